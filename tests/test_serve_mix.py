"""The served workload's request generator and arrival stream (host side, no GPU)."""
import math

import numpy as np

from bsar import scene as S


def test_serve_mix_ranges_and_seeding():
    m = S.serve_mix(256)
    a = S.serve_mix(256)
    assert len(m.requests) == 256 and len(m.dems) == 8
    for r, q in zip(m.requests, a.requests):
        sp = r.spec
        assert 21 <= sp.nx <= 161 and sp.ny == sp.nx and sp.nz == (sp.nx + 1) // 2
        assert 128 <= sp.n_pulses <= 2048
        assert sp.n_samples in (2048, 4096, 8192, 16384)
        assert 5 <= sp.n_scatterers <= 50 and len(r.scat_amp) == sp.n_scatterers
        assert np.all((r.scat_amp >= 0.1) & (r.scat_amp <= 1.0))
        assert 3.0 <= sp.eps_r <= 9.0 and 0.1 <= sp.dem_sigma <= 0.5
        assert r.z.shape == (256, 256)
        assert np.array_equal(r.scat_pos, q.scat_pos) and np.array_equal(r.tx, q.tx)
    # DEMs are shared objects (resident once), each with its sigma
    for (x, y, z, er, sg) in m.dems:
        assert abs(z.std() - sg) < 1e-9
    assert len({id(r.z) for r in m.requests}) <= 8
    # log-uniform grid side: the median side is near the geometric mean of the range
    sides = np.array([r.spec.nx for r in m.requests])
    assert abs(np.median(sides) - math.sqrt(21 * 161)) < 15


def test_poisson_arrivals():
    t = S.poisson_arrivals(20000, 50.0)
    assert t[0] == 0.0 and np.all(np.diff(t) >= 0)
    gaps = np.diff(t)
    assert abs(gaps.mean() - 1 / 50.0) < 0.02 / 50.0 * 10
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.05       # exponential: cv = 1


def test_server_estimate_counts_request_buffers():
    """bsar_server_estimate (host only): the bytes a request reserves grow with its
    pulses x samples (raw + upsampled pulses), its voxels (image and, for small grids, the
    pulse-chunk sums) and its scatterers, and FP16 storage halves the upsampled part."""
    import bsar

    m = S.serve_mix(1, side=(21, 21), pulses=(128, 128), samples_log2=(11, 11), scatterers=(5, 5))
    r = m.requests[0]
    dem = bsar.DemArrays(r.x_vec, r.y_vec, r.z)

    def est(np_=128, ns=2048, nx=21, nscat=5, precision="mixed"):
        tx = np.repeat(r.tx[:1], np_, axis=0)
        gx = 20 + 0.02 * np.arange(nx)
        pos = np.repeat(r.scat_pos[:1], nscat, axis=0)
        return bsar.Server.estimate(dem, tx, tx, gx, gx - 20, gx - 25, n_samples=ns, scat_pos=pos,
                                    scat_amp=np.ones(nscat), precision=precision)

    base = est()
    up = 4
    assert est(np_=256) - base == 128 * (16 * 2048 + 8 * 2048 * up + 48 + 52 + 24 * 5)
    assert est(ns=4096) - base == 128 * (16 * 2048 + 8 * 2048 * up) + 16 * 2048
    # image, plus the pulse-chunk bound of small grids (8 chunk sums per voxel, one count
    # per 128-voxel tile)
    tiles = lambda n: -(-n ** 3 // 128)
    assert est(nx=42) - base == (16 + 128) * (42 ** 3 - 21 ** 3) + 4 * (tiles(42) - tiles(21))
    assert est(nscat=10) - base == 24 * 128 * 5
    assert base - est(precision="mixed_fp16") == 4 * 128 * 2048 * up
