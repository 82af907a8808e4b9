"""The reference arm of bench.py on the CPU: one JSON line with the metric, unit and
workload of the GPU arm, the reference's compiled code timed as the CPU baseline, an e2e
entry with no host-device traffic; under a multi-rank launch only rank 0 prints."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
ARGS = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--config", "1", "--steps", "1",
        "--warmup", "0", "--ref-seconds", "0.5"]


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run(ARGS, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)


@pytest.mark.skipif(not (ROOT / "oracle" / "_ref").exists(), reason="reference harness not built")
def test_reference_arm_line():
    r = _run({})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    sys.path.insert(0, str(ROOT))
    import bench
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 0
    assert d["config"]["workload"].startswith("cfg1-small: 41x41x21 voxels")
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    r = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_parity_sample_covers_the_medium_scene():
    """The medium scene's parity sample: at least 4096 voxels, a uniform sub-lattice plus
    the full 3 x 3 x 3 neighbourhood of each of the 50 scatterers, mapped to the
    reference's flat voxel order (z -> x -> y, y fastest)."""
    import numpy as np
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "c-_bistatic_sar_b200"))
    import bench
    from bsar import scene as S

    sp = S.config_spec(2)
    _, rs, _, _ = S._streams(sp.seed)
    gx, gy, gz = S.grid_axes(sp)
    _, _, sv = S.make_scatterers(sp, rs, gx, gy, gz)
    ii, lat, hoods, groups = bench.parity_sample(sp, sv, 0x5A4B0004)
    assert len(ii) >= 4096 and len(hoods) == 50
    for k, (x, y, z) in enumerate(sv):
        h = ii[groups == k]
        assert len(h) == 27 and (np.abs(h - [x, y, z]).max(axis=1) <= 1).all()
    lat_ii = ii[groups < 0]
    assert len(lat_ii) == len(lat[0]) * len(lat[1]) * len(lat[2])
    v = bench.flat_voxels(sp, ii)
    assert ((v % sp.ny == ii[:, 1]) & ((v // sp.ny) % sp.nx == ii[:, 0]) & (v // (sp.nx * sp.ny) == ii[:, 2])).all()
    # statistics: identical values match exactly; a perturbed copy is measured
    rng = np.random.default_rng(0)
    ref = rng.normal(size=len(ii)) + 1j * rng.normal(size=len(ii))
    st = bench.sample_stats(ref, ref, groups)
    assert st["rel_l2"] == 0.0 and st["argmax_match"] and st["scatterer_argmax_match"] == "50/50"
    st = bench.sample_stats(ref * np.exp(0.002j), ref, groups)
    assert abs(st["max_phase_err_rad"] - 0.002) < 1e-9
