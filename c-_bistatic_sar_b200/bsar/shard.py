"""Multi-GPU partitioning of the voxel grid (one process per GPU).

Voxels are independent and every voxel sums over all pulses, so the image splits into
z-slabs with no exchange during the computation:

* strong: the grid's z axis is cut into `world` contiguous slabs; the slabs are gathered
  (torch.distributed all_gather of the slab images, NCCL over NVLink on GPUs, gloo on CPU)
  into the full image, z fastest, identical to a one-GPU run;
* weak: every rank images a slab of the full grid size, shifted in z by its rank (the
  benchmark's scaling mode).
"""
from __future__ import annotations

import numpy as np


def z_slab(nz: int, rank: int, world: int) -> tuple[int, int]:
    """[begin, end) of rank's contiguous z-slab; sizes differ by at most one."""
    base, extra = divmod(nz, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def weak_slab_axis(gz: np.ndarray, dz: float, rank: int) -> np.ndarray:
    """z axis of rank's slab in weak scaling: the full axis moved down by rank slabs."""
    return np.asarray(gz) - rank * len(gz) * dz


def backproject_sharded(compute, gx, gy, gz, dist=None):
    """Image the grid on all ranks of `dist` (None: one process).

    compute(gx, gy, gz_slab) -> complex image (nx, ny, len(gz_slab)) of this rank's slab.
    Returns the full (nx, ny, nz) image on every rank."""
    import torch

    gz = np.asarray(gz)
    world = dist.get_world_size() if dist else 1
    rank = dist.get_rank() if dist else 0
    b, e = z_slab(len(gz), rank, world)
    part = compute(gx, gy, gz[b:e])
    if not dist:
        return part
    nx, ny = len(gx), len(gy)
    # pad every slab to the largest size so all_gather sees equal shapes
    zmax = z_slab(len(gz), 0, world)[1]
    buf = np.zeros((nx, ny, zmax), dtype=np.complex128)
    buf[:, :, : e - b] = part
    t = torch.from_numpy(buf.view(np.float64).copy())
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = t.to(dev)
    outs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(outs, t)
    full = np.empty((nx, ny, len(gz)), dtype=np.complex128)
    for r, o in enumerate(outs):
        rb, re_ = z_slab(len(gz), r, world)
        full[:, :, rb:re_] = o.cpu().numpy().view(np.complex128)[:, :, : re_ - rb]
    return full


def backproject_scene(ctx, sid, gx, gy, gz, dist=None, **opts):
    """Image of scene `sid` with the grid's z axis split over the ranks of `dist` (strong
    scaling): each rank back-projects its own contiguous z-slab -- one range of the
    reference's flat voxel loop (proc_test_script.cpp:451), through
    ctx.backproject_range with the whole grid's per-pulse anchors -- on its own device,
    with no exchange while imaging, and the slabs are gathered into the full image
    (nx, ny, nz), z fastest, on every rank, equal bit for bit to a one-process run.
    `opts` are ctx.backproject's keywords."""
    nx, ny = len(gx), len(gy)
    nz = len(gz)

    def slab(x, y, z_part):
        # the slab's voxels are the range [b nx ny, e nx ny) of the full grid's order
        world = dist.get_world_size() if dist else 1
        rank = dist.get_rank() if dist else 0
        b, e = z_slab(nz, rank, world)
        full = ctx.backproject_range(sid, gx, gy, gz, b * nx * ny, (e - b) * nx * ny, **opts)
        return full[:, :, b:e]

    return backproject_sharded(slab, gx, gy, gz, dist)
