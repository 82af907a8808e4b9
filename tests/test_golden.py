"""Golden vectors produced by the reference's own compiled code (tests/golden/make_golden.py).

CPU: the oracle restatement reproduces them bit for bit.
GPU: the CUDA library reproduces them through its C ABI -- bit for bit for the DEM,
Fermat and spline functions, to rel-L2 <= 1e-12 for the FFTs and <= 1e-9 for the
back-projection (whose only difference is the device sin/cos); and the full config-1
image of the reference's back-projection (grid search, mean legs) at rel-L2 <= 1e-9 with
the same argmax voxel.
"""
from pathlib import Path

import numpy as np
import pytest

import bsar
from bsar import scene as S
import oracle as O

from conftest import rel_l2

G = np.load(Path(__file__).parent / "golden" / "reference_vectors.npz")
IMG = Path(__file__).parent / "golden" / "cfg1_image.npz"


def test_oracle_reproduces_reference_vectors(oracle):
    dem = O.Dem(G["dem_x"], G["dem_y"], G["dem_z"])
    assert np.array_equal(oracle.dem_elevation(dem, G["xy"]), G["elev"])
    assert np.array_equal(oracle.refraction_points(dem, G["p1"], G["p2"], 1.0, 2.0), G["refr"])
    r, i, v, f = oracle.slant_range_fermat(dem, G["tx"], G["rx"], G["P"], 1.0, 2.0, reflection=True)
    assert np.array_equal(r, G["ranges"]) and np.array_equal(i, G["ida"]) and np.array_equal(v, G["volta"])
    assert np.array_equal(f, G["refl"])
    assert np.array_equal(oracle.spline_upsample(G["sig"][:2, :64], 4), G["spline"])
    assert np.array_equal(np.stack([oracle.fft(s) for s in G["sig"]]), G["fft_f"])
    assert np.array_equal(np.stack([oracle.fft(s, inverse=True) for s in G["sig"]]), G["fft_i"])
    assert np.array_equal(oracle.create_chirp(-25e6, 25e6, 1.3e-6, 60e6), G["chirp"])
    assert np.array_equal(oracle.fft_correlate(G["sig"], G["refv"]), G["corr"])
    assert np.array_equal(oracle.fft_correlate(G["sig"], G["refv"], conj=False), G["conv"])
    n1, n2, c, fs, lam = G["bp_scalars"]
    for legs, key in (("mean", "bp_mean"), ("per", "bp_per")):
        img = oracle.backproject(dem, G["tx"], G["rx"], G["rc"], G["gx"], G["gy"], G["gz"], n1, n2, c, fs, lam,
                                 legs=legs)
        assert np.array_equal(img, G[key])


@pytest.mark.gpu
def test_gpu_reproduces_reference_vectors(ctx):
    dem = bsar.DemArrays(G["dem_x"], G["dem_y"], G["dem_z"])
    assert np.array_equal(ctx.dem_elevation(dem, G["xy"]), G["elev"])
    assert np.array_equal(ctx.refraction_points(dem, G["p1"], G["p2"], 1.0, 2.0), G["refr"])
    r, i, v, f = ctx.slant_range_fermat(dem, G["tx"], G["rx"], G["P"], 1.0, 2.0, reflection=True)
    assert np.array_equal(r, G["ranges"]) and np.array_equal(i, G["ida"]) and np.array_equal(v, G["volta"])
    assert np.array_equal(f, G["refl"])
    assert np.array_equal(ctx.spline_upsample(G["sig"][:2, :64], 4), G["spline"])
    assert rel_l2(ctx.fft(G["sig"]), G["fft_f"]) < 1e-12
    assert rel_l2(ctx.fft(G["sig"], inverse=True), G["fft_i"]) < 1e-12
    assert rel_l2(ctx.fft_correlate(G["sig"], G["refv"]), G["corr"]) < 1e-12
    assert rel_l2(ctx.fft_correlate(G["sig"], G["refv"], conj=False), G["conv"]) < 1e-12
    n1, n2, c, fs, lam = G["bp_scalars"]
    for legs, key in (("mean", "bp_mean"), ("per_pulse", "bp_per")):
        sid = ctx.scene_upload(dem, G["tx"], G["rx"], G["rc"], kind="compressed", upsample=1, n1=n1, n2=n2, c=c,
                               fc=c / lam, fs=fs)
        try:
            img = ctx.backproject(sid, G["gx"], G["gy"], G["gz"], solver="grid", legs=legs, precision="fp64")
        finally:
            ctx.scene_release(sid)
        assert rel_l2(img, G[key]) <= 1e-9


@pytest.mark.gpu
@pytest.mark.skipif(not IMG.exists(), reason="config-1 golden image not generated")
def test_gpu_config1_full_image_matches_reference(ctx):
    g = np.load(IMG)
    sc = S.make_scene(S.config_spec(1))
    import hashlib
    h = hashlib.sha256()
    for a in (sc.x_vec, sc.y_vec, sc.z, sc.tx, sc.rx, sc.raw):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest() == str(g["fingerprint"]), "the seeded config-1 inputs changed since the fixture was made"
    sid = bsar.upload_scene(ctx, sc)
    try:
        img = ctx.backproject(sid, sc.gx, sc.gy, sc.gz, solver="grid", legs="mean", precision="fp64")
    finally:
        ctx.scene_release(sid)
    ref = g["image"]
    assert rel_l2(img, ref) <= 1e-9
    assert np.argmax(np.abs(img)) == np.argmax(np.abs(ref))
