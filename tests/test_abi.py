"""The C-ABI library loads and exports every function include/*.h declares (no GPU
needed), and refuses to run without a device instead of falling back to the CPU."""
import ctypes
import re
from pathlib import Path

import pytest

import bsar

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b(bsar_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    if not bsar.native.LIB_PATH.exists():
        bsar.native.build()
    return bsar.native.lib()


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("bsar_create", "bsar_backproject", "bsar_scene_upload", "bsar_slant_range_fermat",
                 "bsar_spline_upsample", "bsar_fft_correlate", "bsar_dem_elevation"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"libbsar.so lacks {missing}"


def test_status_strings(lib):
    lib.bsar_status_string.restype = ctypes.c_char_p
    for s in range(8):
        assert lib.bsar_status_string(s)


def test_no_cpu_fallback_without_gpu(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(bsar.BsarError):
        bsar.Context(0)
