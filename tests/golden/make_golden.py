"""Generate the golden fixtures from the reference's own compiled functions.

Runs only where the reference tree is present (the objects under oracle/_ref are built
from it by oracle/Makefile).  Writes:

  reference_vectors.npz  small inputs and the reference's outputs for every function on
                         the path: interpolateDEMElevation (in and outside the DEM),
                         calculateRefractionPoint, calculaSlantRangeFermat (ranges,
                         crossings, reflection points), splineInterpolation,
                         FFTProcessor::fft / ifft / fftCorrelation / fftConvolution,
                         createCHIRP, and the inline back-projection of
                         proc_test_script.cpp (mean and per-pulse legs)
  raw_data_vectors.npz   processRawData of the simulator on one target and 6 pulses:
                         the placed deltas (auxData), raw echoes (rawData) and compressed
                         pulses (rootData), with the ranges and radar it ran on
  cfg1_image.npz         the full 41 x 41 x 21 image of the config-1 scene (256 pulses)
                         from the reference's back-projection (grid search, mean legs),
                         with a fingerprint of the generated inputs

Usage: python tests/golden/make_golden.py [--skip-image]
"""
import argparse
import hashlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "c-_bistatic_sar_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

import oracle as O  # noqa: E402
from bsar import scene as S  # noqa: E402


def fingerprint(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def small_vectors(ref: O.Reference):
    rng = np.random.default_rng(20240)
    # DEM 16 x 16 at 0.5 m around (20, 0) with 5 cm roughness
    xv = 20.0 + (np.arange(16) - 7.5) * 0.5
    yv = (np.arange(16) - 7.5) * 0.5
    z = rng.normal(0.0, 0.05, size=(16, 16))
    dem = O.Dem(xv, yv, z)
    xy = np.concatenate([rng.uniform(14.0, 26.0, size=(400, 2)), np.stack([xv[rng.integers(0, 16, 50)],
                                                                           yv[rng.integers(0, 16, 50)]], 1)])
    elev = ref.dem_elevation(dem, xy)
    # 8 pulses of an Archimedean spiral at 30 m, Rx = Tx + (5, 0, 0)
    s = np.arange(8) / 7.0
    tx = np.stack([15 * (1 - s) * np.cos(2 * np.pi * s), 15 * (1 - s) * np.sin(2 * np.pi * s), np.full(8, 30.0)], 1)
    rx = tx + np.array([5.0, 0.0, 0.0])
    p1 = tx[rng.integers(0, 8, 32)]
    p2 = np.stack([rng.uniform(18, 22, 32), rng.uniform(-1.5, 1.5, 32), rng.uniform(-6, -4, 32)], 1)
    refr = ref.refraction_points(dem, p1, p2, 1.0, 2.0)
    P = np.array([20.1, -0.3, -5.2])
    ranges, ida, volta, refl = ref.slant_range_fermat(dem, tx, rx, P, 1.0, 2.0)
    # signal functions
    sig = rng.normal(size=(3, 256)) + 1j * rng.normal(size=(3, 256))
    spline = ref.spline_upsample(sig[:2, :64], 4)
    fft_f = np.stack([ref.fft(r) for r in sig])
    fft_i = np.stack([ref.fft(r, inverse=True) for r in sig])
    chirp = ref.create_chirp(-25e6, 25e6, 1.3e-6, 60e6)        # the reference's default radar
    refv = np.zeros(256, complex)
    half = len(chirp) // 2
    refv[: len(chirp) - half] = chirp[half:]
    refv[256 - half:] = chirp[:half]
    corr = ref.fft_correlate(sig, refv, conj=True)
    conv = ref.fft_correlate(sig, refv, conj=False)
    # back-projection on a 4 x 3 x 2 grid over the 8 pulses
    rc = rng.normal(size=(8, 1024)) + 1j * rng.normal(size=(8, 1024))
    gx = np.array([19.9, 20.0, 20.1, 20.2])
    gy = np.array([-0.1, 0.0, 0.1])
    gz = np.array([-5.1, -4.9])
    # fs_eff / lambda chosen so the delays land inside the 1024-sample pulses
    bp_args = dict(n1=1.0, n2=2.0, c=3e8, fs_eff=3.0e9, lam=0.3)
    bp_mean = ref.backproject(dem, tx, rx, rc, gx, gy, gz, legs="mean", **bp_args)
    bp_per = ref.backproject(dem, tx, rx, rc, gx, gy, gz, legs="per", **bp_args)
    return dict(dem_x=xv, dem_y=yv, dem_z=z, xy=xy, elev=elev, tx=tx, rx=rx, p1=p1, p2=p2, refr=refr, P=P,
                ranges=ranges, ida=ida, volta=volta, refl=refl, sig=sig, spline=spline, fft_f=fft_f, fft_i=fft_i,
                chirp=chirp, refv=refv, corr=corr, conv=conv, rc=rc, gx=gx, gy=gy, gz=gz, bp_mean=bp_mean,
                bp_per=bp_per, bp_scalars=np.array([bp_args[k] for k in ("n1", "n2", "c", "fs_eff", "lam")]))


def raw_vectors(ref: O.Reference, orc: O.Oracle):
    """The simulator's processRawData (src/raw_data_processing.cpp:292-452) for one target
    over 6 pulses, on ranges from the FP64 Newton crossings of the oracle (the solver the
    GPU echo synthesis runs, bit for bit): the placed deltas, the raw echoes and the
    compressed pulses, 1024 samples each."""
    rng = np.random.default_rng(20241)
    n = 32
    xv = 20.0 + (np.arange(n) - (n - 1) / 2.0) * 0.25
    yv = (np.arange(n) - (n - 1) / 2.0) * 0.25
    z = rng.normal(0.0, 0.04, size=(n, n))
    dem = O.Dem(xv, yv, z)
    s = np.arange(6) / 5.0
    tx = np.stack([15 * (1 - s) * np.cos(2 * np.pi * s), 15 * (1 - s) * np.sin(2 * np.pi * s), np.full(6, 30.0)], 1)
    rx = tx + np.array([5.0, 0.0, 0.0])
    P = np.array([20.05, -0.12, -5.03])
    n1, n2, c, fc, fs, f0, f1, T, M, rcs = 1.0, 2.0, 3e8, 1e9, 1.2e9, -250e6, 250e6, 1e-7, 1024, 0.8
    W = S.search_nodes_for(xv, yv)
    Pn = np.repeat(P[None], len(tx), 0)
    a = orc.refraction_points(dem, tx, Pn, n1, n2, solver="newton", search_nodes=W)
    b = orc.refraction_points(dem, Pn, rx, n2, n1, solver="newton", search_nodes=W)

    def dist(u, w):
        # the synthesis kernel's distance: sqrt(x*x + y*y + z*z) of u - w, in that order
        return np.array([float(np.sqrt((p[0] - q[0]) * (p[0] - q[0]) + (p[1] - q[1]) * (p[1] - q[1])
                                       + (p[2] - q[2]) * (p[2] - q[2]))) for p, q in zip(u, w)])

    ranges = np.stack([dist(tx, a), dist(Pn, a), dist(rx, b), dist(Pn, b)])    # r1Tx, r2Tx, r1Rx, r2Rx
    assert np.all(np.isfinite(ranges)) and np.all(ranges > 0)
    aux, raw, root, chirp = ref.process_raw_data(tx, rx, P, ranges, f0, f1, T, fs, c / fc, rcs, c, M, n1, n2)
    return dict(raw_dem_x=xv, raw_dem_y=yv, raw_dem_z=z, raw_tx=tx, raw_rx=rx, raw_P=P, raw_ranges=ranges,
                raw_scalars=np.array([n1, n2, c, fc, fs, f0, f1, T, M, rcs]), raw_aux=aux, raw_raw=raw,
                raw_root=root, raw_chirp=chirp)


def cfg1_image(ref: O.Reference):
    spec = S.config_spec(1)
    sc = S.make_scene(spec)
    dem = O.Dem(sc.x_vec, sc.y_vec, sc.z)
    rc = ref.spline_upsample(ref.fft_correlate(sc.raw, sc.reference), spec.upsample)
    img = ref.backproject(dem, sc.tx, sc.rx, rc, sc.gx, sc.gy, sc.gz, spec.n1, spec.n2, 3e8, sc.fs_eff, sc.lam,
                          legs="mean", nthreads=0)
    return dict(image=img, fingerprint=np.array(fingerprint(sc.x_vec, sc.y_vec, sc.z, sc.tx, sc.rx, sc.raw)),
                gx=sc.gx, gy=sc.gy, gz=sc.gz, scat_voxel=sc.scat_voxel)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--skip-image", action="store_true")
    args = ap.parse_args()
    O.build(ref=True)
    if not O.Reference.available():
        sys.exit("the reference tree is needed to build oracle/_ref")
    ref = O.Reference()
    np.savez_compressed(HERE / "reference_vectors.npz", **small_vectors(ref))
    print("wrote", HERE / "reference_vectors.npz")
    np.savez_compressed(HERE / "raw_data_vectors.npz", **raw_vectors(ref, O.Oracle()))
    print("wrote", HERE / "raw_data_vectors.npz")
    if not args.skip_image:
        np.savez_compressed(HERE / "cfg1_image.npz", **cfg1_image(ref))
        print("wrote", HERE / "cfg1_image.npz")


if __name__ == "__main__":
    main()
