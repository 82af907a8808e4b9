"""Multi-rank partitioning on CPU: two gloo ranks image their z-slabs and gather the
full image, equal to a one-process run; weak-scaling slabs tile the depth axis; the
max-over-ranks timing reduction takes the slowest rank."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from bsar import shard


def _fake_compute(gx, gy, gz):
    X, Y, Z = np.meshgrid(gx, gy, gz, indexing="ij")
    return np.exp(1j * (3 * X + 5 * Y)) * (1 + Z)


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        gx, gy, gz = np.linspace(0, 1, 4), np.linspace(-1, 1, 3), np.linspace(-6, -4, 7)
        img = shard.backproject_sharded(_fake_compute, gx, gy, gz, dist)
        t = torch.tensor([float(rank + 1)])
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        q.put((rank, img, float(t.item())))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_z_slabs_partition_the_axis():
    for nz in (1, 7, 81, 128):
        for world in (1, 2, 3, 8):
            spans = [shard.z_slab(nz, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == nz
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [e - b for b, e in spans]
            assert max(sizes) - min(sizes) <= 1


def test_weak_slabs_stack_in_depth():
    gz = -5.0 + (np.arange(81) - 40) * 0.02
    s1 = shard.weak_slab_axis(gz, 0.02, 1)
    assert np.allclose(s1[-1] + 0.02, gz[0])


def test_two_gloo_ranks_gather_the_full_image():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    gx, gy, gz = np.linspace(0, 1, 4), np.linspace(-1, 1, 3), np.linspace(-6, -4, 7)
    want = _fake_compute(gx, gy, gz)
    for rank, img, tmax in res:
        assert np.array_equal(img, want)
        assert tmax == 2.0


def _scene():
    from bsar import scene as S
    # 64 pulses (fewer than 256: no pulse chunks, so slabs and the full grid sum alike)
    return S.make_scene(S.scaled(S.config_spec(2), n_pulses=64, n_samples=4096, nx=24, ny=20, nz=9, n_scatterers=3))


def _library_worker(rank, world, port, q):
    import torch.distributed as dist

    import bsar
    from bsar import shard as sh

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sc = _scene()
        with bsar.Context(0) as ctx:
            sid = bsar.upload_scene(ctx, sc)
            out = {}
            for prec in ("fp64", "mixed"):
                out[prec] = sh.backproject_scene(ctx, sid, sc.gx, sc.gy, sc.gz, dist, solver="newton",
                                                 legs="per_pulse", precision=prec)
            ctx.scene_release(sid)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_two_ranks_run_the_library_on_their_slabs():
    """Two processes (gloo ranks, both on cuda:0) each run libbsar on their z-slab; the
    gathered FP64 Newton and mixed images equal the one-process images bit for bit."""
    import bsar

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_library_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    sc = _scene()
    with bsar.Context(0) as c:
        sid = bsar.upload_scene(c, sc)
        want = {prec: c.backproject(sid, sc.gx, sc.gy, sc.gz, solver="newton", legs="per_pulse", precision=prec)
                for prec in ("fp64", "mixed")}
        c.scene_release(sid)
    for rank, out in res:
        for prec in want:
            assert np.array_equal(out[prec], want[prec]), (rank, prec)
