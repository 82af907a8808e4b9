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
