"""Continuous-batching server (bsar_server_* of the C ABI).

* every request's image is the same, bit for bit, alone on the server, in a mix of
  other requests, over many small batches, with and without CUDA-graph replay, and
  through the one-request entry point (bsar_backproject, mixed form);
* the served mixed images meet the mixed-form bounds against the plain FP64 Newton
  image (rel-L2 <= 1e-3, max phase error <= 0.01 rad, same argmax voxel);
* admission honours the HBM budget: a request above the whole budget fails alone,
  requests that do not fit together wait for each other;
* a request that fails at admission does not disturb the others.
"""
import numpy as np
import pytest

import bsar
from bsar import scene as S

from conftest import max_phase_err, rel_l2

pytestmark = pytest.mark.gpu


def _mix(n, seed=11, **kw):
    # up to 320 pulses: the small grids with 256 or more run in pulse chunks
    args = dict(side=(9, 25), pulses=(32, 320), samples_log2=(11, 12), scatterers=(3, 8))
    args.update(kw)
    return S.serve_mix(n, seed=S.SEED_BASE + seed, n_dems=3, **args)


def _submit(srv, sc, **kw):
    return bsar.submit_scene(srv, sc, sc.gx, sc.gy, sc.gz, **kw)


def _direct(ctx, sc, precision):
    sid = bsar.synthesize_scene(ctx, sc)
    try:
        return ctx.backproject(sid, sc.gx, sc.gy, sc.gz, solver="newton", legs="per_pulse", precision=precision)
    finally:
        ctx.scene_release(sid)


@pytest.fixture(scope="module")
def mix():
    return _mix(6)


@pytest.fixture(scope="module")
def served(ctx, mix):
    """Request 0 alone, then all requests submitted at once."""
    with bsar.Server(ctx, max_inflight=8) as srv:
        alone, _ = srv.wait(_submit(srv, mix.requests[0]))
        ids = [_submit(srv, sc) for sc in mix.requests]
        imgs = [srv.wait(i)[0] for i in ids]
        st = srv.stats()
    return alone, imgs, st


def test_same_alone_and_in_mix(served):
    alone, imgs, st = served
    assert np.array_equal(alone, imgs[0])
    assert st["completed"] == 7 and st["failed"] == 0
    assert st["peak_inflight"] >= 2
    # batches were on the device for part of the span from first submission to last image
    assert 0 < st["batch_busy_s"] <= st["busy_s"] + 1e-3


def test_served_equals_one_request_entry_point(ctx, mix, served):
    _, imgs, _ = served
    for sc, img in zip(mix.requests, imgs):
        assert np.array_equal(img, _direct(ctx, sc, "mixed"))


def test_served_meets_mixed_bounds(ctx, mix, served):
    _, imgs, _ = served
    for sc, img in zip(mix.requests, imgs):
        ref = _direct(ctx, sc, "fp64")
        assert rel_l2(img, ref) <= 1e-3
        assert max_phase_err(img, ref) <= 0.01
        assert np.argmax(np.abs(img)) == np.argmax(np.abs(ref))


@pytest.mark.parametrize("opts", [dict(tiles_per_launch=5), dict(use_graph=False), dict(max_inflight=1)])
def test_batching_does_not_change_results(ctx, mix, served, opts):
    _, imgs, _ = served
    with bsar.Server(ctx, **opts) as srv:
        ids = [_submit(srv, sc) for sc in mix.requests[:4]]
        got = [srv.wait(i)[0] for i in ids]
        st = srv.stats()
    for a, b in zip(got, imgs[:4]):
        assert np.array_equal(a, b)
    if "tiles_per_launch" in opts:
        assert st["launches"] >= st["tiles"] // 5
    if opts.get("max_inflight") == 1:
        assert st["peak_inflight"] == 1


def test_fp16_storage_served(ctx, mix):
    sc = mix.requests[1]
    with bsar.Server(ctx) as srv:
        img, lat = srv.wait(_submit(srv, sc, precision="mixed_fp16"))
    assert lat > 0
    assert np.array_equal(img, _direct(ctx, sc, "mixed_fp16"))
    ref = _direct(ctx, sc, "fp64")
    assert rel_l2(img, ref) <= 1e-3


def _estimate(sc):
    dem = bsar.DemArrays(sc.x_vec, sc.y_vec, sc.z)
    return bsar.Server.estimate(dem, sc.tx, sc.rx, sc.gx, sc.gy, sc.gz, n_samples=sc.spec.n_samples,
                                scat_pos=sc.scat_pos, scat_amp=sc.scat_amp)


def test_budget_serialises_requests(ctx):
    m = _mix(4, seed=12, side=(15, 15), pulses=(48, 48), samples_log2=(11, 11))
    e = max(_estimate(sc) for sc in m.requests)
    with bsar.Server(ctx, hbm_budget_bytes=int(1.5 * e)) as srv:
        ids = [_submit(srv, sc) for sc in m.requests]
        imgs = [srv.wait(i)[0] for i in ids]
        st = srv.stats()
    assert st["completed"] == 4 and st["peak_inflight"] == 1
    assert st["peak_reserved_bytes"] <= int(1.5 * e)
    with bsar.Server(ctx, hbm_budget_bytes=int(4.5 * e)) as srv:
        ids = [_submit(srv, sc) for sc in m.requests]
        imgs2 = [srv.wait(i)[0] for i in ids]
        st = srv.stats()
    assert st["peak_inflight"] >= 2
    for a, b in zip(imgs, imgs2):
        assert np.array_equal(a, b)


def test_request_above_budget_fails_alone(ctx):
    m = _mix(2, seed=13, side=(11, 11), pulses=(40, 40), samples_log2=(11, 11))
    big = S.scaled(m.requests[0].spec, n_pulses=400)
    sc_big = S.Scene(big, m.requests[0].x_vec, m.requests[0].y_vec, m.requests[0].z, *S.make_trajectories(big),
                     m.requests[0].gx, m.requests[0].gy, m.requests[0].gz, m.requests[0].scat_pos,
                     m.requests[0].scat_amp, m.requests[0].scat_voxel)
    budget = (_estimate(sc_big) + _estimate(m.requests[1])) // 2
    assert _estimate(m.requests[1]) < budget < _estimate(sc_big)
    with bsar.Server(ctx, hbm_budget_bytes=budget) as srv:
        i_big = _submit(srv, sc_big)
        i_ok = _submit(srv, m.requests[1])
        with pytest.raises(bsar.BsarError) as e:
            srv.wait(i_big)
        assert e.value.status == 2
        img, _ = srv.wait(i_ok)
        st = srv.stats()
    assert st["failed"] == 1 and st["completed"] == 1
    assert np.array_equal(img, _direct(ctx, m.requests[1], "mixed"))


def test_bad_request_isolated(ctx, mix):
    sc = mix.requests[2]
    z_bad = sc.z.copy()
    z_bad[3, 4] = np.nan
    bad = S.Scene(sc.spec, sc.x_vec, sc.y_vec, z_bad, sc.tx, sc.rx, sc.gx, sc.gy, sc.gz, sc.scat_pos, sc.scat_amp,
                  sc.scat_voxel)
    with bsar.Server(ctx) as srv:
        i_bad = _submit(srv, bad)
        i_ok = _submit(srv, mix.requests[3])
        with pytest.raises(bsar.BsarError) as e:
            srv.wait(i_bad)
        assert e.value.status == 1
        img, _ = srv.wait(i_ok)
    assert np.array_equal(img, _direct(ctx, mix.requests[3], "mixed"))


def test_unsupported_precision_rejected_at_submit(ctx, mix):
    with bsar.Server(ctx) as srv:
        with pytest.raises(bsar.BsarError) as e:
            _submit(srv, mix.requests[0], precision="fp64")
        assert e.value.status == 6


def test_requests_on_dems_of_different_spacing_share_the_server(ctx):
    """Requests whose DEM spacings need different node-scan widths (0.25 m: 13 x 13 nodes,
    0.5 m: 7 x 7) are in flight together; every image equals the one-request image."""
    reqs = []
    for k, (d, n) in enumerate([(0.25, 256), (0.5, 128), (0.25, 256), (0.5, 128)]):
        spec = S.scaled(S.config_spec(2), nx=17, ny=15, nz=4, n_pulses=96, n_samples=2048, dem_d=d, dem_n=n,
                        n_scatterers=3, seed=S.SEED_BASE + 300 + k)
        reqs.append(S.make_scene(spec, with_raw=False))
    assert {S.search_nodes_for(r.x_vec, r.y_vec) for r in reqs} == {3, 6}
    with bsar.Server(ctx, max_inflight=4) as srv:
        ids = [_submit(srv, sc) for sc in reqs]
        imgs = [srv.wait(i)[0] for i in ids]
    for sc, img in zip(reqs, imgs):
        assert np.array_equal(img, _direct(ctx, sc, "mixed"))
