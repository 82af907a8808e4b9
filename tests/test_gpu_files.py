"""Pulse files into resident scenes and device images out to files, through the C ABI:
the simulator's matrix file read as the imager reads it, or in its own row-major layout
(transposed on the GPU), must give the same scene as an upload of the same pulses; a
device image written with the GPU permute must equal the host writer's file byte for
byte, and the reference's export3DComplexMatrix file."""
import numpy as np
import pytest

import bsar
from bsar import scene as S

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sc():
    return S.make_scene(S.scaled(S.config_spec(1), n_pulses=24, nx=7, ny=9, nz=5, dxy=0.16, dz=0.32))


@pytest.fixture(scope="module")
def compressed(sc, oracle):
    return oracle.fft_correlate(sc.raw, sc.reference)       # (Np, Ns) complex128


def _upload_args(sc):
    sp = sc.spec
    return dict(upsample=sp.upsample, n1=sp.n1, n2=sp.n2, c=3e8, fc=sp.fc, fs=sp.fs)


@pytest.mark.parametrize("layout", ["as_imager", "row_major"])
def test_scene_from_file_equals_upload(ctx, sc, compressed, tmp_path, layout):
    np_, ns = compressed.shape
    p = tmp_path / f"rootData_{layout}.bin"
    if layout == "as_imager":
        # the imager indexes element (r, p) at p*Ns + r of a file whose dims are (Ns, Np)
        flat = compressed.reshape(-1)
        dims = (ns, np_)
        bsar.native.matrix_write(p, flat.reshape(dims))
    else:
        bsar.native.matrix_write(p, compressed.T)             # row-major [range][pulse]
    dem = bsar.DemArrays(sc.x_vec, sc.y_vec, sc.z)
    a = ctx.scene_upload_file(dem, sc.tx, sc.rx, p, layout=layout, **_upload_args(sc))
    b = ctx.scene_upload(dem, sc.tx, sc.rx, compressed, kind="compressed", **_upload_args(sc))
    try:
        assert np.array_equal(ctx.scene_read_samples(a, np_, ns), compressed)
        ia = ctx.backproject(a, sc.gx, sc.gy, sc.gz, solver="grid", legs="mean", precision="fp64")
        ib = ctx.backproject(b, sc.gx, sc.gy, sc.gz, solver="grid", legs="mean", precision="fp64")
        assert np.array_equal(ia, ib)
    finally:
        ctx.scene_release(a)
        ctx.scene_release(b)


def test_scene_from_file_rejects_pulse_count_mismatch(ctx, sc, compressed, tmp_path):
    p = tmp_path / "rd.bin"
    bsar.native.matrix_write(p, compressed.T)
    dem = bsar.DemArrays(sc.x_vec, sc.y_vec, sc.z)
    with pytest.raises(bsar.BsarError) as e:
        ctx.scene_upload_file(dem, sc.tx[:-1], sc.rx[:-1], p, layout="row_major", **_upload_args(sc))
    assert e.value.status == 1


def test_device_image_file_matches_host_and_reference(ctx, reference, tmp_path):
    import torch

    rng = np.random.default_rng(7)
    nx, ny, nz = 37, 45, 33                         # not multiples of the 32 x 32 tile
    img = rng.normal(size=(nx, ny, nz)) + 1j * rng.normal(size=(nx, ny, nz))
    gx, gy, gz = np.arange(nx) * 0.02, np.arange(ny) * 0.02 - 0.4, np.arange(nz) * 0.05 - 5
    d = torch.from_numpy(img.view(np.float64).reshape(-1).copy()).cuda()
    ctx.image_export_device(tmp_path / "dev.bin", d.data_ptr(), nx, ny, nz, gx, gy, gz)
    bsar.native.image_export(tmp_path / "host.bin", img, gx, gy, gz)
    reference.export_3d(tmp_path / "ref.bin", img, gx, gy, gz)
    dev = (tmp_path / "dev.bin").read_bytes()
    assert dev == (tmp_path / "host.bin").read_bytes() == (tmp_path / "ref.bin").read_bytes()
    for ax in "xyz":
        assert (tmp_path / f"dev_grid_{ax}.csv").read_bytes() == (tmp_path / f"ref_grid_{ax}.csv").read_bytes()


def test_file_round_trip_of_backprojected_image(ctx, sc, tmp_path):
    sid = bsar.upload_scene(ctx, sc)
    try:
        img = ctx.backproject(sid, sc.gx, sc.gy, sc.gz, solver="newton", legs="per_pulse", precision="mixed")
    finally:
        ctx.scene_release(sid)
    bsar.native.image_export(tmp_path / "out.bin", img)
    v, dims, cplx = bsar.native.matrix_read(tmp_path / "out.bin")
    back = v.reshape(dims[::-1]).transpose(2, 1, 0)
    assert cplx and rel_l2(back, img) == 0.0
