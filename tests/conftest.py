"""Test configuration: import paths, the `gpu` marker and shared fixtures.

GPU tests (``-m gpu``) call the CUDA library through its C ABI and compare with the
oracle (oracle/, test infrastructure).  CPU tests (``-m "not gpu"``) cover the oracle
against the reference's own code and committed golden vectors, the host logic and the
library's exported symbols.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "c-_bistatic_sar_b200"))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.build(ref=True)
    return O.Oracle()


@pytest.fixture(scope="session")
def reference():
    import oracle as O
    O.build(ref=True)
    if not O.Reference.available():
        pytest.skip("reference objects (oracle/_ref) not built: the reference tree is absent")
    return O.Reference()


@pytest.fixture(scope="session")
def ctx():
    import bsar
    if not bsar.native.LIB_PATH.exists():
        bsar.native.build()
    c = bsar.Context(0)
    yield c
    c.close()


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def max_phase_err(img, ref, floor=1e-3):
    m = np.abs(ref) >= floor * np.abs(ref).max()
    return float(np.abs(np.angle(img[m] * np.conj(ref[m]))).max()) if m.any() else 0.0
