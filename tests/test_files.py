"""Files around the path against the reference's own readers and writers (compiled
under oracle/_ref): the binary matrix format (src/binary_reader.cpp,
src/data_export.cpp), the 3-D image file with its grid CSVs, and the ESRI ASCII DEM
loader (src/load_dem_simple.cpp).  Host code only: no GPU needed."""
import numpy as np
import pytest

import bsar


def _bytes(p):
    return open(p, "rb").read()


@pytest.fixture(scope="module")
def rng():
    return np.random.default_rng(0x5A4B00F1)


def test_matrix_file_bytes_match_reference(reference, tmp_path, rng):
    m = rng.normal(size=(7, 5)) + 1j * rng.normal(size=(7, 5))
    bsar.native.matrix_write(tmp_path / "ours.bin", m)
    reference.export_complex_matrix(tmp_path / "ref.bin", m)
    assert _bytes(tmp_path / "ours.bin") == _bytes(tmp_path / "ref.bin")
    v, dims, cplx = bsar.native.matrix_read(tmp_path / "ref.bin")
    assert dims == [7, 5] and cplx and np.array_equal(v, m.ravel())
    v2, dims2, cplx2 = reference.read_binary(tmp_path / "ours.bin")
    assert dims2 == [7, 5] and cplx2 and np.array_equal(v2, m.ravel())


def test_real_and_higher_rank_files(reference, tmp_path, rng):
    r = rng.normal(size=(3, 4, 2))
    bsar.native.matrix_write(tmp_path / "real.bin", r)
    v, dims, cplx = bsar.native.matrix_read(tmp_path / "real.bin")
    assert dims == [3, 4, 2] and not cplx
    assert np.array_equal(v.real, r.ravel()) and not v.imag.any()
    v2, dims2, cplx2 = reference.read_binary(tmp_path / "real.bin")
    assert dims2 == dims and not cplx2 and np.array_equal(v2, v)


def test_truncated_and_missing_files(reference, tmp_path, rng):
    m = rng.normal(size=(6, 6)) + 0j
    bsar.native.matrix_write(tmp_path / "m.bin", m)
    data = _bytes(tmp_path / "m.bin")
    for cut in (3, 20, 40, len(data) - 8):
        p = tmp_path / f"cut{cut}.bin"
        p.write_bytes(data[:cut])
        with pytest.raises(bsar.BsarError):
            bsar.native.matrix_read(p)
        with pytest.raises(RuntimeError):
            reference.read_binary(p)
    with pytest.raises(bsar.BsarError) as e:
        bsar.native.matrix_read(tmp_path / "absent.bin")
    assert e.value.status == 5


def test_empty_matrix_is_not_written(tmp_path):
    with pytest.raises(bsar.BsarError):
        bsar.native.matrix_write(tmp_path / "e.bin", np.zeros((0, 4), complex))
    assert not (tmp_path / "e.bin").exists()


def test_image_file_and_grid_csvs_match_reference(reference, tmp_path, rng):
    img = rng.normal(size=(5, 4, 3)) + 1j * rng.normal(size=(5, 4, 3))
    gx, gy, gz = 19.2 + 0.04 * np.arange(5), -0.8 + 0.04 * np.arange(4), -5.8 + 0.08 * np.arange(3)
    bsar.native.image_export(tmp_path / "ours.bin", img, gx, gy, gz)
    reference.export_3d(tmp_path / "ref.bin", img, gx, gy, gz)
    assert _bytes(tmp_path / "ours.bin") == _bytes(tmp_path / "ref.bin")
    for ax in "xyz":
        assert _bytes(tmp_path / f"ours_grid_{ax}.csv") == _bytes(tmp_path / f"ref_grid_{ax}.csv")
    v, dims, _ = bsar.native.matrix_read(tmp_path / "ours.bin")
    assert dims == [5, 4, 3]
    assert np.array_equal(v.reshape(3, 4, 5).transpose(2, 1, 0), img)      # x fastest in the file


ESRI = {
    "plain": "ncols 4\nnrows 3\nxllcorner 10.0\nyllcorner -2.5\ncellsize 0.5\nNODATA_value -9999\n"
             "1 2 3 4\n5 6 7 8\n9 10 11 12\n",
    "missing_values": "ncols 4\nnrows 3\nxllcorner 0\nyllcorner 0\ncellsize 2\nnodata_value -1\n"
                      "1 2\n3 4 5 6\n7 x 9 10\n",
    "blank_before_data": "ncols 3\nnrows 2\ncellsize 1\n\n1 2 3\n4 5 6\n",
    "extra_rows": "ncols 2\nnrows 2\n1 2\n3 4\n5 6\n7 8\n",
    "short_rows": "ncols 3\nnrows 4\nxllcorner 1\nyllcorner 2\ncellsize 0.25\n1 2 3\n4 5 6\n",
    "unknown_key": "ncols 2\nnrows 2\nxllcenter 5\n1 2\n3 4\n",
    "no_header": "1.5 2.5\n3.5 4.5\n",
}


@pytest.mark.parametrize("name", sorted(ESRI))
def test_esri_dem_matches_reference(reference, tmp_path, name):
    p = tmp_path / f"{name}.asc"
    p.write_text(ESRI[name])
    x, y, z, flags = bsar.native.dem_load_esri(p)
    rx, ry, rz = reference.load_dem(p)
    assert np.array_equal(x, rx) and np.array_equal(y, ry) and np.array_equal(z, rz)
    assert bool(flags & 4) == (name in ("short_rows", "no_header"))      # rows read != nrows


def test_esri_fallback_dem(reference, tmp_path):
    for p in (tmp_path / "terrain.tif", tmp_path / "absent.asc"):
        if p.suffix == ".tif":
            p.write_text("not a grid")
        x, y, z, flags = bsar.native.dem_load_esri(p)
        rx, ry, rz = reference.load_dem(p)
        assert x.shape == (32,) and np.array_equal(x, rx) and np.array_equal(y, ry) and np.array_equal(z, rz)
        assert flags == (1 if p.suffix == ".tif" else 2)
