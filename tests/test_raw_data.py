"""The simulator's echo model, processRawData (src/raw_data_processing.cpp:292-452),
against golden vectors from the reference's own compiled function (one target, 6 pulses,
1024-sample pulses, ranges from FP64 Newton crossings; tests/golden/make_golden.py).

CPU: a driver built against the reference's headers and linked with its compiled sources
reproduces the golden auxData / rawData / rootData bit for bit (the driver itself is right).
GPU: the same driver built against include/bsar_compat.h (processRawData's GPU shim) and
the on-device echo synthesis with the simulator's bins (bsar_scene_synthesize_ex,
BSAR_SYNTH_REFERENCE_BINS; it solves the same crossings itself) reproduce them to
rel-L2 <= 1e-12.
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import bsar
import oracle as O

from conftest import rel_l2

ROOT = Path(__file__).resolve().parent.parent
LIB = ROOT / "c-_bistatic_sar_b200" / "lib"
DRIVER = ROOT / "tests" / "compat" / "raw_driver.cpp"
G = np.load(ROOT / "tests" / "golden" / "raw_data_vectors.npz")
n1, n2, c, fc, fs, f0, f1, T, M, rcs = G["raw_scalars"]
M = int(M)
NP = len(G["raw_tx"])


def _input_file(path: Path):
    with open(path, "wb") as f:
        np.array([NP, M], dtype=np.int64).tofile(f)
        for a in (G["raw_tx"], G["raw_rx"], G["raw_P"], G["raw_ranges"]):
            np.ascontiguousarray(a, dtype=np.float64).tofile(f)
        np.array([f0, f1, T, fs, c / fc, rcs, c, n1, n2], dtype=np.float64).tofile(f)


def _run_driver(tmp_path: Path, compat: bool):
    exe = tmp_path / ("raw_compat" if compat else "raw_ref")
    if compat:
        if not (LIB / "libbsar_compat.so").exists():
            bsar.native.build()
        cmd = ["/usr/bin/g++", "-O1", "-std=c++17", "-DUSE_BSAR_HEADER", f"-I{ROOT / 'include'}", str(DRIVER),
               f"-L{LIB}", "-lbsar_compat", f"-Wl,-rpath,{LIB}", "-o", str(exe)]
    else:
        ref_dir = O.REF_SO.parent
        cmd = ["/usr/bin/g++", "-O1", "-std=c++17", f"-I{O.REF_TREE / 'include'}", str(DRIVER), str(O.REF_SO),
               f"-Wl,-rpath,{ref_dir}", "-fopenmp", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    _input_file(tmp_path / "in.bin")
    subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], check=True, capture_output=True,
                   timeout=300)
    out = np.fromfile(tmp_path / "out.bin", dtype=np.complex128).reshape(3, NP, M)
    return out[0], out[1], out[2]


@pytest.mark.skipif(not (O.REF_SO.exists() and (O.REF_TREE / "include").exists()),
                    reason="the reference's headers and compiled sources are needed")
def test_reference_driver_reproduces_golden(tmp_path):
    aux, raw, root = _run_driver(tmp_path, compat=False)
    assert np.array_equal(aux, G["raw_aux"])
    assert np.array_equal(raw, G["raw_raw"])
    assert np.array_equal(root, G["raw_root"])


def test_golden_echo_sits_at_the_simulators_bin():
    """Each pulse's delta sits at 1 + round(t fs) with t the two-way optical path / c
    (:322-361), with rcs * exp(-j 2 pi L / lambda)."""
    r1t, r2t, r1r, r2r = G["raw_ranges"]
    L = n1 * r1t + n2 * r2t + n1 * r1r + n2 * r2r
    bins = 1 + np.round(L / c * fs).astype(int)
    for i in range(NP):
        nz = np.flatnonzero(G["raw_aux"][i])
        assert list(nz) == [bins[i]]
        assert abs(G["raw_aux"][i, bins[i]] - rcs * np.exp(-2j * np.pi / (c / fc) * L[i])) < 1e-12


@pytest.mark.gpu
def test_compat_shim_reproduces_golden(tmp_path):
    aux, raw, root = _run_driver(tmp_path, compat=True)
    assert rel_l2(aux, G["raw_aux"]) <= 1e-15
    assert rel_l2(raw, G["raw_raw"]) <= 1e-12
    assert rel_l2(root, G["raw_root"]) <= 1e-12


@pytest.mark.gpu
def test_gpu_echo_synthesis_reproduces_golden(ctx):
    """One scatterer of amplitude rcs at the golden target, no noise, simulator bins: the
    synthesised raw pulses equal rawData and, compressed in FP64 with no upsampling,
    rootData."""
    dem = bsar.DemArrays(G["raw_dem_x"], G["raw_dem_y"], G["raw_dem_z"])
    sid = ctx.scene_synthesize(dem, G["raw_tx"], G["raw_rx"], M, G["raw_P"][None], np.array([rcs]),
                               snr_db=float("inf"), seed=0, upsample=1, n1=n1, n2=n2, c=c, fc=fc, fs=fs,
                               chirp_f0=f0, chirp_f1=f1, chirp_T=T, reference_bins=True)
    try:
        raw = ctx.scene_read_samples(sid, NP, M)
        ctx.scene_compress(sid, "fp64")
        root = ctx.scene_read_stored(sid, NP, M, "fp64")
    finally:
        ctx.scene_release(sid)
    assert rel_l2(raw, G["raw_raw"]) <= 1e-12
    assert rel_l2(root, G["raw_root"]) <= 1e-12
