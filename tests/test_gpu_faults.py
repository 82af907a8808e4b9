"""Failure handling with no GPU fault, hang or trap: every failure here is a bounded wait
that runs out by design, or a request the caller withdraws.

* the mixed kernel's bounded wait for its DEM tile copy (limit 0: every wait runs out at
  once) reports BSAR_ERR_TIMEOUT, and the image is still the tiled run's, bit for bit,
  because the fallback reads the same heights from global memory; the next call with the
  default limit succeeds (a 25 x 25 node scan, the width whose kernel stages the tile);
* a server whose batch time limit is shorter than any batch stops: its requests fail with
  BSAR_ERR_TIMEOUT, later submissions are refused, destroying it waits for the batch on
  the device, and the context serves a new server normally afterwards;
* a cancelled request completes with BSAR_ERR_CANCELLED while the rest of the mix is
  unchanged bit for bit.

The reference's own failure surface is thrown I/O errors and silent fallbacks
(proc_test_script.cpp:225, 898-901); these are the serving and device-wait counterparts.
"""
import numpy as np
import pytest

import bsar
from bsar import scene as S

pytestmark = pytest.mark.gpu

TIMEOUT, CANCELLED, NOT_FOUND = 3, 8, 5


@pytest.fixture(scope="module")
def scene():
    return S.make_scene(S.scaled(S.config_spec(2), n_pulses=64, n_samples=4096, nx=24, ny=24, nz=3, n_scatterers=3))


def _mix(n, seed=23):
    return S.serve_mix(n, seed=S.SEED_BASE + seed, n_dems=2, side=(9, 21), pulses=(32, 96), samples_log2=(11, 12),
                       scatterers=(2, 5))


def _submit(srv, sc):
    return bsar.submit_scene(srv, sc, sc.gx, sc.gy, sc.gz)


def _direct(ctx, sc):
    sid = bsar.synthesize_scene(ctx, sc)
    try:
        return ctx.backproject(sid, sc.gx, sc.gy, sc.gz, solver="newton", legs="per_pulse", precision="mixed")
    finally:
        ctx.scene_release(sid)


# 3 m on the 0.25 m DEM: 12 nodes each side
WIDE = dict(solver="newton", legs="per_pulse", precision="mixed", search_radius_m=3.0)


def test_tile_wait_that_runs_out_reports_timeout_with_the_same_image(scene):
    with bsar.Context(0) as ctx:
        sid = bsar.upload_scene(ctx, scene)
        try:
            ref = ctx.backproject(sid, scene.gx, scene.gy, scene.gz, **WIDE)
            ctx.set_tile_wait_limit(0)
            out = np.zeros_like(ref)
            with pytest.raises(bsar.BsarError) as e:
                ctx.backproject(sid, scene.gx, scene.gy, scene.gz, out=out, **WIDE)
            assert e.value.status == TIMEOUT
            assert np.array_equal(out, ref)
            ctx.set_tile_wait_limit(-1)
            again = ctx.backproject(sid, scene.gx, scene.gy, scene.gz, **WIDE)
            assert np.array_equal(again, ref)
        finally:
            ctx.scene_release(sid)


def test_server_batch_time_limit_stops_the_server():
    mix = _mix(3)
    with bsar.Context(0) as ctx:
        with bsar.Server(ctx, batch_timeout_s=1e-7) as srv:
            ids = [_submit(srv, sc) for sc in mix.requests]
            for i in ids:
                with pytest.raises(bsar.BsarError) as e:
                    srv.wait(i, timeout_s=120.0)
                assert e.value.status == TIMEOUT
            with pytest.raises(bsar.BsarError) as e:
                _submit(srv, mix.requests[0])
            assert e.value.status == TIMEOUT
            assert srv.stats()["failed"] == 3
        # destroyed after its batch finished on the device; the context works on
        with bsar.Server(ctx) as srv:
            img, _ = srv.wait(_submit(srv, mix.requests[1]), timeout_s=120.0)
        assert np.array_equal(img, _direct(ctx, mix.requests[1]))


@pytest.mark.parametrize("which", [0, 3])
def test_cancelled_request_fails_alone(ctx, which):
    mix = _mix(5, seed=29)
    with bsar.Server(ctx, max_inflight=2) as srv:
        ids = [_submit(srv, sc) for sc in mix.requests]
        srv.cancel(ids[which])
        with pytest.raises(bsar.BsarError) as e:
            srv.wait(ids[which], timeout_s=120.0)
        assert e.value.status == CANCELLED
        imgs = {i: srv.wait(rid, timeout_s=120.0)[0] for i, rid in enumerate(ids) if i != which}
        with pytest.raises(bsar.BsarError) as e:
            srv.cancel(ids[(which + 1) % 5])          # already finished
        assert e.value.status == NOT_FOUND
        with pytest.raises(bsar.BsarError) as e:
            srv.cancel(987654)
        assert e.value.status == NOT_FOUND
        st = srv.stats()
    assert st["completed"] == 4 and st["failed"] == 1
    for i, img in imgs.items():
        assert np.array_equal(img, _direct(ctx, mix.requests[i]))
