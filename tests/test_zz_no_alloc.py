"""bsar_backproject_mixed_noalloc, the entry point for callers that cannot allocate GPU
memory (another allocator owns it, or a cudaFree's device-wide wait is not allowed):
its image must equal the allocating entry point bsar_backproject's, on two calls in a
row that share the fixed per-device scratch array."""
import numpy as np
import pytest

import bsar
from bsar import scene as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    return S.make_scene(S.scaled(S.config_spec(2), n_pulses=40, n_samples=4096, nx=13, ny=11, nz=6, dxy=0.1,
                                 dz=0.1, n_scatterers=4))


@pytest.fixture(scope="module")
def chunked_scene():
    # small grid, 256 pulses: both entry points run it in pulse chunks
    return S.make_scene(S.scaled(S.config_spec(2), n_pulses=256, n_samples=4096, nx=13, ny=11, nz=6, dxy=0.1,
                                 dz=0.1, n_scatterers=4))


def _device_free_bytes() -> int:
    """cudaMemGetInfo's free bytes of device 0 (the driver's view, not a pool's)."""
    import torch
    return int(torch.cuda.mem_get_info(0)[0])


def _alloc(ctx, sid, gx, gy, gz, precision):
    return ctx.backproject(sid, gx, gy, gz, solver="newton", legs="per_pulse", precision=precision)


@pytest.mark.parametrize("which", ["scene", "chunked_scene"])
@pytest.mark.parametrize("precision", ["mixed", "mixed_fp16"])
def test_noalloc_matches_allocating_entry_point(ctx, which, precision, request):
    scene = request.getfixturevalue(which)
    sid = bsar.upload_scene(ctx, scene)
    try:
        ctx.scene_compress(sid, precision)
        ref = _alloc(ctx, sid, scene.gx, scene.gy, scene.gz, precision)
        used = ctx.bytes_in_use
        first = ctx.backproject_mixed_noalloc(sid, scene.gx, scene.gy, scene.gz, precision=precision)
        # the first call may load the scratch's module; after it the device's free memory
        # must not move (an allocation outside the context's pool would show here)
        free_before = _device_free_bytes()
        second = ctx.backproject_mixed_noalloc(sid, scene.gx, scene.gy, scene.gz, precision=precision)
        free_after = _device_free_bytes()
        assert ctx.bytes_in_use == used
        assert abs(free_after - free_before) < (1 << 20), (free_before, free_after)
    finally:
        ctx.scene_release(sid)
    assert np.array_equal(first, ref)
    assert np.array_equal(second, ref)


def test_noalloc_two_grids_in_a_row(ctx, scene):
    """A second call on another grid reuses the scratch: counter, status and image are
    reset, nothing of the first call leaks into the second."""
    gx2 = scene.gx[2:9] + 0.013
    gz2 = scene.gz[:4] - 0.05
    sid = bsar.upload_scene(ctx, scene)
    try:
        ctx.scene_compress(sid, "mixed")
        a = ctx.backproject_mixed_noalloc(sid, scene.gx, scene.gy, scene.gz)
        b = ctx.backproject_mixed_noalloc(sid, gx2, scene.gy, gz2)
        ra = _alloc(ctx, sid, scene.gx, scene.gy, scene.gz, "mixed")
        rb = _alloc(ctx, sid, gx2, scene.gy, gz2, "mixed")
    finally:
        ctx.scene_release(sid)
    assert np.array_equal(a, ra)
    assert np.array_equal(b, rb)


def test_noalloc_requires_compressed_scene(ctx, scene):
    sid = bsar.upload_scene(ctx, scene)
    try:
        used = ctx.bytes_in_use
        with pytest.raises(bsar.BsarError) as e:
            ctx.backproject_mixed_noalloc(sid, scene.gx, scene.gy, scene.gz)
        assert e.value.status == 1 and "bsar_scene_compress" in str(e.value)
        assert ctx.bytes_in_use == used
    finally:
        ctx.scene_release(sid)


def test_noalloc_rejects_grid_beyond_scratch(ctx, scene):
    sid = bsar.upload_scene(ctx, scene)
    try:
        ctx.scene_compress(sid, "mixed")
        gx = 20.0 + 0.01 * np.arange(200)
        gz = -5.0 + 0.01 * np.arange(120)
        with pytest.raises(bsar.BsarError) as e:
            ctx.backproject_mixed_noalloc(sid, gx, gx - 20.0, gz)
        assert e.value.status == 1 and "scratch" in str(e.value)
    finally:
        ctx.scene_release(sid)


def test_noalloc_rejects_fp64(ctx, scene):
    sid = bsar.upload_scene(ctx, scene)
    try:
        keep, g = ctx._grid(scene.gx, scene.gy, scene.gz)
        out = np.empty((len(scene.gx), len(scene.gy), len(scene.gz)), dtype=np.complex128)
        o = bsar.native.BpOpts(1, 1, 0, 0, 0.0)          # Newton, per-pulse, FP64
        st = ctx.L.bsar_backproject_mixed_noalloc(ctx.h, sid, bsar.native.C.byref(g), bsar.native.C.byref(o),
                                                  bsar.native._p(out.view(np.float64)))
        assert st == 6
    finally:
        ctx.scene_release(sid)
