"""Device memory of a context.

A context takes its buffers from its own stream-ordered pool, which keeps freed blocks
for later calls. Repeated scene upload -> compression -> back-projection -> release
cycles must hand every buffer back (bytes_in_use comes back to the same value once the
context's caches are filled) and give the same image every time, because a reused block
holds a previous call's data.
A second context, with a pool of its own, must give the same image too.
"""
import numpy as np
import pytest

import bsar
from bsar import scene as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sc():
    return S.make_scene(S.scaled(S.config_spec(2), n_pulses=32, n_samples=4096, nx=12, ny=10, nz=4, dxy=0.1,
                                 dz=0.1, n_scatterers=4))


def _cycle(ctx, sc, precision):
    sid = bsar.upload_scene(ctx, sc)
    try:
        return ctx.backproject(sid, sc.gx, sc.gy, sc.gz, solver="newton", legs="per_pulse", precision=precision)
    finally:
        ctx.scene_release(sid)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_repeated_cycles_release_buffers_and_repeat_the_image(ctx, sc, precision):
    # the first cycle may fill the context's caches (twiddles, grid axes, status word)
    first = _cycle(ctx, sc, precision)
    used = ctx.bytes_in_use
    for _ in range(3):
        assert np.array_equal(_cycle(ctx, sc, precision), first)
        assert ctx.bytes_in_use == used


def test_second_context_gives_the_same_image(ctx, sc):
    want = _cycle(ctx, sc, "mixed")
    with bsar.Context(0) as other:
        assert np.array_equal(_cycle(other, sc, "mixed"), want)
        used = other.bytes_in_use
        assert np.array_equal(_cycle(other, sc, "mixed"), want)
        assert other.bytes_in_use == used
