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
