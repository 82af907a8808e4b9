"""GPU back-projection through the C ABI against the oracle.

* plain FP64 form, grid solver (the reference's algorithm), mean or per-pulse legs:
  rel-L2 <= 1e-9 and the same argmax voxel as the oracle restatement of
  proc_test_script.cpp:451-767;
* plain FP64 Newton form against the oracle's FP64 Newton: rel-L2 <= 1e-9;
* mixed forms against the plain FP64 Newton image: rel-L2 <= 1e-3, max phase error
  <= 0.01 rad, same argmax voxel.
"""
import numpy as np
import pytest

import bsar
from bsar import scene as S
import oracle as O

from conftest import max_phase_err, rel_l2

pytestmark = pytest.mark.gpu


def _setup(spec):
    sc = S.make_scene(spec)
    return sc


@pytest.fixture(scope="module")
def small():
    # config-1 geometry, fewer pulses and voxels so the CPU oracle finishes in seconds
    return _setup(S.scaled(S.config_spec(1), n_pulses=40, nx=9, ny=9, nz=5, dxy=0.16, dz=0.32))


@pytest.fixture(scope="module")
def chunked():
    # 405 voxels (4 tiles) and 256 pulses: the mixed kernel runs each tile in 2 pulse chunks
    return _setup(S.scaled(S.config_spec(1), n_pulses=256, nx=9, ny=9, nz=5, dxy=0.16, dz=0.32))


@pytest.fixture(scope="module")
def rough():
    return _setup(S.scaled(S.config_spec(2), n_pulses=48, n_samples=4096, nx=11, ny=11, nz=6, dxy=0.1, dz=0.1,
                           n_scatterers=4))


@pytest.fixture(scope="module")
def large():
    # config-5 DEM and signal (1024^2 fBm at 0.125 m, so a 25 x 25 node scan; 16384
    # samples), a 10 x 40 x 4 grid so warps span y
    return _setup(S.scaled(S.config_spec(5), n_pulses=48, nx=10, ny=40, nz=4, n_scatterers=6))


def _oracle_image(oracle, sc, legs, solver):
    sp = sc.spec
    dem = O.Dem(sc.x_vec, sc.y_vec, sc.z)
    rc = oracle.spline_upsample(oracle.fft_correlate(sc.raw, sc.reference), sp.upsample)
    return oracle.backproject(dem, sc.tx, sc.rx, rc, sc.gx, sc.gy, sc.gz, sp.n1, sp.n2, 3e8, sc.fs_eff, sc.lam,
                              legs="mean" if legs == "mean" else "per", solver=solver,
                              search_nodes=S.search_nodes_for(sc.x_vec, sc.y_vec))


@pytest.mark.parametrize("legs", ["mean", "per_pulse"])
def test_plain_grid_matches_reference_algorithm(ctx, oracle, small, legs):
    sid = bsar.upload_scene(ctx, small)
    try:
        img = ctx.backproject(sid, small.gx, small.gy, small.gz, solver="grid", legs=legs, precision="fp64")
    finally:
        ctx.scene_release(sid)
    ref = _oracle_image(oracle, small, legs, "grid")
    assert rel_l2(img, ref) <= 1e-9
    assert np.argmax(np.abs(img)) == np.argmax(np.abs(ref))


@pytest.mark.parametrize("which", ["small", "rough", "large"])
def test_plain_newton_matches_oracle(ctx, oracle, which, request):
    sc = request.getfixturevalue(which)
    sid = bsar.upload_scene(ctx, sc)
    try:
        img = ctx.backproject(sid, sc.gx, sc.gy, sc.gz, solver="newton", legs="per_pulse", precision="fp64")
    finally:
        ctx.scene_release(sid)
    ref = _oracle_image(oracle, sc, "per_pulse", "newton")
    assert rel_l2(img, ref) <= 1e-9
    assert np.argmax(np.abs(img)) == np.argmax(np.abs(ref))


@pytest.mark.parametrize("precision", ["mixed", "mixed_fp16"])
@pytest.mark.parametrize("which", ["small", "chunked", "rough", "large"])
def test_mixed_matches_fp64(ctx, which, precision, request):
    sc = request.getfixturevalue(which)
    sid = bsar.upload_scene(ctx, sc)
    try:
        ref = ctx.backproject(sid, sc.gx, sc.gy, sc.gz, solver="newton", legs="per_pulse", precision="fp64")
        img = ctx.backproject(sid, sc.gx, sc.gy, sc.gz, solver="newton", legs="per_pulse", precision=precision)
    finally:
        ctx.scene_release(sid)
    assert rel_l2(img, ref) <= 1e-3
    assert max_phase_err(img, ref) <= 0.01
    assert np.argmax(np.abs(img)) == np.argmax(np.abs(ref))


@pytest.fixture(scope="module")
def inverted():
    # antennas 60 m below the terrain and voxels straddling it: the node scan's height
    # term a_z Z + |N - G| falls with height for nodes below a voxel, so its lower bound
    # does not hold and nothing may be pruned
    sc = _setup(S.scaled(S.config_spec(2), n_pulses=48, n_samples=4096, nx=11, ny=11, nz=3, dxy=0.1,
                         n_scatterers=4))
    sc.tx = sc.tx.copy()
    sc.rx = sc.rx.copy()
    sc.tx[:, 2] -= 60.0
    sc.rx[:, 2] -= 60.0
    sc.gz = np.array([-0.4, 0.0, 0.4])
    return sc


@pytest.fixture(scope="module")
def slab():
    # medium-scene geometry (256^2 fBm DEM at 0.25 m, eps_r 6) on a 48 x 48 x 3 slab with
    # 256 consecutive pulses: whole warps of neighbouring voxels, consecutive pulses
    return _setup(S.scaled(S.config_spec(2), n_pulses=256, n_samples=4096, nx=48, ny=48, nz=3, n_scatterers=5))


@pytest.mark.parametrize("precision", ["mixed", "mixed_fp16"])
@pytest.mark.parametrize("which", ["small", "chunked", "rough", "large", "slab", "inverted"])
def test_pruned_node_scan_is_bit_identical(ctx, which, precision, request):
    """The mixed node scan skips rows and column groups that its lower bound excludes; the
    image must be bit for bit the one of the scan that ranks every node."""
    sc = request.getfixturevalue(which)
    sid = bsar.upload_scene(ctx, sc)
    try:
        full = ctx.backproject(sid, sc.gx, sc.gy, sc.gz, solver="newton", legs="per_pulse", precision=precision,
                               exhaustive=True)
        pruned = ctx.backproject(sid, sc.gx, sc.gy, sc.gz, solver="newton", legs="per_pulse", precision=precision)
    finally:
        ctx.scene_release(sid)
    assert np.array_equal(pruned, full)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("which", ["chunked", "rough"])
def test_voxel_ranges_add_up_to_the_image(ctx, which, precision, request):
    """bsar_backproject_range: three ranges of the flat voxel order, each with the whole
    grid's anchors and pulse chunks, add up to bsar_backproject's image bit for bit."""
    sc = request.getfixturevalue(which)
    kw = dict(solver="newton", legs="per_pulse", precision=precision)
    nv = len(sc.gx) * len(sc.gy) * len(sc.gz)
    cuts = [0, nv // 3, (2 * nv) // 3 + 5, nv]
    sid = bsar.upload_scene(ctx, sc)
    try:
        full = ctx.backproject(sid, sc.gx, sc.gy, sc.gz, **kw)
        parts = [ctx.backproject_range(sid, sc.gx, sc.gy, sc.gz, a, b - a, **kw) for a, b in zip(cuts, cuts[1:])]
        with pytest.raises(bsar.BsarError):
            ctx.backproject_range(sid, sc.gx, sc.gy, sc.gz, nv - 3, 5, **kw)
    finally:
        ctx.scene_release(sid)
    assert np.array_equal(parts[0] + parts[1] + parts[2], full)
    flat = np.zeros(nv, dtype=bool)
    flat[cuts[1]:cuts[2]] = True
    zi, rem = np.divmod(np.arange(nv), len(sc.gx) * len(sc.gy))
    xi, yi = np.divmod(rem, len(sc.gy))
    mask = np.zeros(full.shape, dtype=bool)
    mask[xi[flat], yi[flat], zi[flat]] = True
    assert np.all(parts[1][~mask] == 0) and np.array_equal(parts[1][mask], full[mask])


def test_unknown_backprojection_flags_are_rejected(ctx, small):
    sid = bsar.upload_scene(ctx, small)
    try:
        keep, g = ctx._grid(small.gx, small.gy, small.gz)
        out = np.empty((len(small.gx), len(small.gy), len(small.gz)), dtype=np.complex128)
        o = bsar.native.BpOpts(1, 1, 1, 2, 0.0)          # Newton, per-pulse, mixed, flag bit 1
        st = ctx.L.bsar_backproject(ctx.h, sid, bsar.native.C.byref(g), bsar.native.C.byref(o),
                                    bsar.native._p(out.view(np.float64)))
        assert st == 1
    finally:
        ctx.scene_release(sid)


@pytest.mark.parametrize("which", ["chunked"])
def test_mixed_small_grid_pulse_chunks_are_deterministic(ctx, which, request):
    """Grids too small to fill the GPU run each 128-voxel tile's pulses in chunks; the
    last chunk of a tile to finish adds the chunks in chunk order.  Whatever order the
    chunks finish in, repeated runs give the same bits, through the device-buffer entry
    point as well as the host one."""
    import torch

    sc = request.getfixturevalue(which)
    sid = bsar.upload_scene(ctx, sc)
    try:
        imgs = [ctx.backproject(sid, sc.gx, sc.gy, sc.gz, solver="newton", legs="per_pulse", precision="mixed")
                for _ in range(4)]
        nv = len(sc.gx) * len(sc.gy) * len(sc.gz)
        d = torch.empty((nv, 2), dtype=torch.float64, device="cuda")
        ctx.backproject_device(sid, sc.gx, sc.gy, sc.gz, d.data_ptr(), solver="newton", legs="per_pulse",
                               precision="mixed")
        ctx.synchronize()
        dev = d.cpu().numpy().view(np.complex128).reshape(imgs[0].shape)
    finally:
        ctx.scene_release(sid)
    for img in imgs[1:] + [dev]:
        assert np.array_equal(img, imgs[0])


def test_scatterer_focuses_at_its_voxel(ctx):
    spec = S.scaled(S.config_spec(1), n_pulses=64, nx=15, ny=15, nz=9, dxy=0.04, dz=0.08, n_scatterers=1,
                    snr_db=np.inf)
    sc = S.make_scene(spec)
    sid = bsar.upload_scene(ctx, sc)
    try:
        img = ctx.backproject(sid, sc.gx, sc.gy, sc.gz, solver="newton", legs="per_pulse", precision="mixed")
    finally:
        ctx.scene_release(sid)
    ix, iy, iz = np.unravel_index(np.argmax(np.abs(img)), img.shape)
    assert (ix, iy, iz) == tuple(sc.scat_voxel[0])


def test_invalid_requests_are_rejected(ctx, small):
    sid = bsar.upload_scene(ctx, small)
    try:
        with pytest.raises(bsar.BsarError) as e:
            ctx.backproject(sid, small.gx, small.gy, small.gz, solver="grid", legs="per_pulse", precision="mixed")
        assert e.value.status == 6
        with pytest.raises(bsar.BsarError) as e:
            ctx.backproject(sid, [], small.gy, small.gz)
        assert e.value.status == 1
    finally:
        ctx.scene_release(sid)
    with pytest.raises(bsar.BsarError) as e:
        ctx.backproject(987654, small.gx, small.gy, small.gz)
    assert e.value.status == 5
    tx = small.tx.copy()
    tx[3, 1] = np.nan
    with pytest.raises(bsar.BsarError) as e:
        ctx.scene_upload(bsar.DemArrays(small.x_vec, small.y_vec, small.z), tx, small.rx, small.raw,
                         chirp_T=1e-6, chirp_f0=-2.5e8, chirp_f1=2.5e8)
    assert e.value.status == 1
