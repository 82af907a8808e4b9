"""Several host threads on one context.

The imager calls calculaSlantRangeFermat from up to 12 OpenMP threads at once
(proc_test_script.cpp:428,451,484): through the C++ drop-in layer those calls must give
the same results as serial calls, bit for bit.  Through the C ABI, threads that share a
context each read their own failure from bsar_last_error, and an empty message after a
success, while other threads' calls fail and succeed in between.
"""
import subprocess
import threading
from pathlib import Path

import numpy as np
import pytest

import bsar

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
LIB = ROOT / "c-_bistatic_sar_b200" / "lib"


def test_compat_fermat_from_12_openmp_threads(tmp_path):
    if not (LIB / "libbsar_compat.so").exists():
        bsar.native.build()
    exe = tmp_path / "threads"
    subprocess.run(["/usr/bin/g++", "-O1", "-std=c++17", "-fopenmp", "-DUSE_BSAR_HEADER", f"-I{ROOT / 'include'}",
                    str(ROOT / "tests" / "compat" / "threads_driver.cpp"), f"-L{LIB}", "-lbsar_compat",
                    f"-Wl,-rpath,{LIB}", "-o", str(exe)], check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=600).stdout.split()
    got = dict(zip(out[::2], map(int, out[1::2])))
    assert got["voxels"] == 96 and got["threads"] == 12
    assert got["differ"] == 0 and got["failed"] == 0


def test_last_error_is_per_thread(ctx):
    dem = bsar.DemArrays(np.arange(4) * 0.5, np.arange(3) * 0.5, np.zeros((3, 4)))
    xy = np.array([[0.7, 0.2]])
    errors = []

    def worker(t):
        try:
            for i in range(100):
                sid = 10**12 + 1000 * t + i              # never a live scene id
                try:
                    ctx.scene_release(sid)
                    errors.append(f"thread {t}: release of unknown id {sid} succeeded")
                except bsar.BsarError as e:
                    if e.status != 5 or f"unknown scene id {sid}" not in str(e):
                        errors.append(f"thread {t}: got '{e}' for id {sid}")
                ctx.dem_elevation(dem, xy)
                if ctx.last_error() != "":
                    errors.append(f"thread {t}: message '{ctx.last_error()}' after a success")
        except Exception as e:                           # noqa: BLE001 -- reported below
            errors.append(f"thread {t}: {e!r}")

    ts = [threading.Thread(target=worker, args=(t,)) for t in range(8)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert errors == []


def test_last_error_not_inherited_by_a_later_context():
    """A thread's failure on a context that another thread then destroys is not reported
    for a context created afterwards, even one that reuses the freed address."""
    a = bsar.Context(0)
    seen, ctxs = {}, {"a": a}
    failed, swapped = threading.Event(), threading.Event()

    def worker():
        try:
            a.scene_release(10**12 + 7)
        except bsar.BsarError:
            pass
        seen["a"] = a.last_error()
        failed.set()
        swapped.wait(60)
        seen["b"] = ctxs["b"].last_error()          # same thread, the new context

    t = threading.Thread(target=worker)
    t.start()
    failed.wait(60)
    a.close()
    ctxs["b"] = bsar.Context(0)
    swapped.set()
    t.join()
    try:
        assert "unknown scene id" in seen["a"]
        assert seen["b"] == ""
    finally:
        ctxs["b"].close()
