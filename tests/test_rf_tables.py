"""Host-built tables of the FP32 register transforms (k_pulse_compress_rf, 4096-16384
points; kernels.hpp): the lane-ordered twiddles of the second and fourth passes and the
stored order of the matched-filter spectrum.  The kernels read entry e of each where the
natural layout had the value the formulas below name, so a wrong map would change every
compressed sample; the GPU tests check the samples against the oracle, this checks the
maps themselves on the host.

A P-point transform (P = 2^L) runs as T = P/16 threads of 16 elements; the second and
fourth passes work on blocks of B = 16 TB elements and the third on groups of TB,
TB = 2^(L-12).
"""
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
DRIVER = Path(__file__).parent / "compat" / "rf_tables_driver.cpp"
CUDA_INC = Path("/usr/local/cuda/include")


def _tables(tmp_path):
    exe = tmp_path / "rf_tables"
    subprocess.run(["/usr/bin/g++", "-O1", "-std=c++17", f"-I{ROOT / 'c-_bistatic_sar_b200' / 'csrc'}",
                    f"-I{ROOT / 'include'}", f"-I{CUDA_INC}", str(DRIVER), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    lines = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    out = {}
    for k in range(3):
        head = lines[2 * k].split()
        L, n = int(head[0]), int(head[1])
        tw = np.array(head[2:], dtype=np.int64)
        assert len(tw) == n
        out[L] = (tw, np.array(lines[2 * k + 1].split(), dtype=np.int64))
    return out


def test_second_pass_twiddles_in_lane_order(tmp_path):
    for L, (tw, _) in _tables(tmp_path).items():
        P, TB = 1 << L, 1 << (L - 12)
        B = 16 * TB
        assert len(tw) == 15 * B
        # the stage of span d (8, 4, 2, 1), butterfly k < d, lane r < B: the twiddle the
        # natural-order table holds at (r + B k) P / (2 B d), the one that pass needs
        for d in (8, 4, 2, 1):
            for k in range(d):
                r = np.arange(B)
                assert np.array_equal(tw[B * (16 - 2 * d) + B * k + r], (r + B * k) * (P // (2 * B * d)))
        assert tw.min() >= 0 and tw.max() < P // 2


def test_spectrum_in_third_pass_order(tmp_path):
    for L, (_, spec) in _tables(tmp_path).items():
        P, T, TB = 1 << L, 1 << (L - 4), 1 << (L - 12)
        B = 16 * TB
        # a permutation: every spectrum entry stored once
        assert np.array_equal(np.sort(spec), np.arange(P))
        # element m of thread t, stored at m T + t, is the one the third pass multiplies:
        # group t / TB, offset t mod TB + TB m
        m, t = np.divmod(np.arange(P), T)
        assert np.array_equal(spec, (t // TB) * B + t % TB + TB * m)
