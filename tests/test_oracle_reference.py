"""The C restatement (oracle/bsar_oracle.c) against the reference's own compiled
functions (oracle/_ref): bit-exact on seeded inputs, including out-of-DEM points."""
import numpy as np
import pytest

from bsar import scene as S
import oracle as O


@pytest.fixture(scope="module")
def small():
    spec = S.scaled(S.config_spec(1), n_pulses=16, n_samples=2048, nx=5, ny=4, nz=3)
    return S.make_scene(spec)


def test_dem_elevation_bitexact(oracle, reference, small):
    dem = O.Dem(small.x_vec, small.y_vec, small.z)
    rng = np.random.default_rng(7)
    xy = np.concatenate([
        rng.uniform(-20, 60, size=(3000, 2)),                                 # inside and far outside
        np.stack([small.x_vec[rng.integers(0, 64, 300)], small.y_vec[rng.integers(0, 64, 300)]], 1),  # on nodes
        np.array([[np.nan, 0.0], [20.0, np.nan], [np.inf, 1.0], [small.x_vec[-1], small.y_vec[0]]]),
    ])
    a = oracle.dem_elevation(dem, xy)
    b = reference.dem_elevation(dem, xy)
    assert np.array_equal(a, b, equal_nan=True)


def test_dem_edge_cases(oracle, reference):
    # descending axis, single-node axis, empty DEM
    for xv, yv in (([3.0, 2.0, 1.0], [0.0, 1.0]), ([1.0], [0.0, 1.0, 2.0]), ([0.0, 1.0], [5.0])):
        z = np.arange(len(xv) * len(yv), dtype=float).reshape(len(yv), len(xv)) * 0.1
        dem = O.Dem(xv, yv, z)
        xy = np.random.default_rng(1).uniform(-1, 4, size=(400, 2))
        assert np.array_equal(oracle.dem_elevation(dem, xy), reference.dem_elevation(dem, xy))
    empty = O.Dem([], [], np.zeros(0))
    assert np.all(oracle.dem_elevation(empty, [[1.0, 2.0]]) == 0.0)


def test_slant_range_fermat_bitexact(oracle, reference, small):
    dem = O.Dem(small.x_vec, small.y_vec, small.z)
    sp = small.spec
    for P in ([20.0, 0.1, -5.0], [19.3, -0.7, -4.3]):
        a = oracle.slant_range_fermat(dem, small.tx, small.rx, P, sp.n1, sp.n2, reflection=True)
        b = reference.slant_range_fermat(dem, small.tx, small.rx, P, sp.n1, sp.n2)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def test_spline_fft_chirp_bitexact(oracle, reference, small):
    raw = small.raw[:3]
    assert np.array_equal(oracle.spline_upsample(raw), reference.spline_upsample(raw))
    assert np.array_equal(oracle.fft(raw[0]), reference.fft(raw[0]))
    assert np.array_equal(oracle.fft(raw[0], True), reference.fft(raw[0], True))
    assert np.array_equal(oracle.fft_correlate(raw, small.reference), reference.fft_correlate(raw, small.reference))
    assert np.array_equal(oracle.fft_correlate(raw, small.reference, conj=False),
                          reference.fft_correlate(raw, small.reference, conj=False))
    sp = small.spec
    c1 = oracle.create_chirp(-sp.bandwidth / 2, sp.bandwidth / 2, sp.pulse_T, sp.fs)
    c2 = reference.create_chirp(-sp.bandwidth / 2, sp.bandwidth / 2, sp.pulse_T, sp.fs)
    assert np.array_equal(c1, c2)
    # the non-power-of-two FFT leaves data unchanged in both
    x = raw[0][:100]
    assert np.array_equal(oracle.fft(x), x) and np.array_equal(reference.fft(x), x)


@pytest.mark.parametrize("legs", ["mean", "per_pulse"])
def test_backproject_bitexact(oracle, reference, small, legs):
    sp = small.spec
    dem = O.Dem(small.x_vec, small.y_vec, small.z)
    rc = oracle.spline_upsample(oracle.fft_correlate(small.raw, small.reference))
    kw = dict(legs="mean" if legs == "mean" else "per")
    a = oracle.backproject(dem, small.tx, small.rx, rc, small.gx, small.gy, small.gz, sp.n1, sp.n2, 3e8,
                           small.fs_eff, small.lam, **kw)
    b = reference.backproject(dem, small.tx, small.rx, rc, small.gx, small.gy, small.gz, sp.n1, sp.n2, 3e8,
                              small.fs_eff, small.lam, **kw)
    assert np.array_equal(a, b)


def test_newton_not_worse_than_grid(oracle, small):
    """On the smooth config-1 DEM the Newton crossing never has a longer optical path
    than the reference's grid search."""
    sp = small.spec
    dem = O.Dem(small.x_vec, small.y_vec, small.z)
    W = S.search_nodes_for(small.x_vec, small.y_vec)
    for P in ([20.0, 0.1, -5.0], [19.5, 0.6, -4.5], [20.7, -0.7, -5.7]):
        g = oracle.slant_range_fermat(dem, small.tx, small.rx, P, sp.n1, sp.n2, solver="grid")[0]
        n = oracle.slant_range_fermat(dem, small.tx, small.rx, P, sp.n1, sp.n2, solver="newton", search_nodes=W)[0]
        Lg = sp.n1 * g[0] + sp.n2 * g[1] + sp.n2 * g[3] + sp.n1 * g[2]
        Ln = sp.n1 * n[0] + sp.n2 * n[1] + sp.n2 * n[3] + sp.n1 * n[2]
        assert np.all(Ln <= Lg + 1e-12)


def test_numpy_synthesis_solver_matches_oracle_newton(oracle):
    spec = S.scaled(S.config_spec(2), n_pulses=32)
    sc = S.make_scene(spec, with_raw=False)
    dem = O.Dem(sc.x_vec, sc.y_vec, sc.z)
    W = S.search_nodes_for(sc.x_vec, sc.y_vec)
    rng = np.random.default_rng(3)
    P = np.stack([rng.choice(sc.gx, 64), rng.choice(sc.gy, 64), rng.choice(sc.gz, 64)], 1)
    A = sc.tx[rng.integers(0, 32, 64)]
    a = oracle.refraction_points(dem, A, P, spec.n1, spec.n2, solver="newton", search_nodes=W)
    b = S.fermat_newton(sc.x_vec, sc.y_vec, sc.z, A, P, spec.n1, spec.n2)
    assert np.array_equal(a, b)
