"""Seeded synthetic bistatic SAR scenes.

No public dataset is involved: every input is generated here from a seed.

* DEM: a plane plus i.i.d. Gaussian roughness, or an fBm surface made by spectral
  synthesis (|H(k)| ~ k^(-beta/2), random phase, rescaled to the requested sigma).
  Rows follow y (z[j, i] = height at (x_vec[i], y_vec[j])), as Z_DEM in the reference.
* Trajectories: Archimedean spiral r = r_max (1 - s), theta = 2 pi turns s,
  s = i / (Np - 1), at constant altitude; Rx = Tx + (5, 0, 0) m.
* Scatterers: point targets snapped to voxel centres of the imaging grid.
* Echoes: for each pulse and scatterer, the refracted two-way optical path
  L = n1 r1Tx + n2 r2Tx + n2 r2Rx + n1 r1Rx (per-pulse legs, Newton Fermat solve) gives
  tau = L / c; the raw pulse is sum_s a_s exp(-j 2 pi f_c tau_s) chirp(t - tau_s) with the
  chirp centred on tau (the reference's convention, src/raw_data_processing.cpp:380-421,
  but at the exact fractional delay).  Complex Gaussian noise is added with
  SNR = peak compressed-echo power of a unit scatterer / compressed noise power
  = Nc / sigma^2 (Nc = chirp length).
* Seeds: 0x5A4B0000 + config; sub-streams for dem / scatterers / noise / requests are
  spawned from one SeedSequence.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

import numpy as np

C_LIGHT = 3e8  # the reference's VelocidadeLuz, src/radar_init.cpp:74
SEED_BASE = 0x5A4B0000


@dataclass
class SceneSpec:
    name: str
    # imaging grid
    nx: int
    ny: int
    nz: int
    dxy: float
    dz: float
    center: tuple = (20.0, 0.0, -5.0)
    # DEM
    dem_n: int = 64
    dem_d: float = 0.5
    dem_kind: str = "plane"          # "plane" (iid roughness) | "fbm"
    dem_sigma: float = 0.03
    dem_beta: float = 2.0
    eps_r: float = 4.0
    # trajectory
    n_pulses: int = 256
    r_max: float = 15.0
    turns: float = 3.0
    altitude: float = 30.0
    rx_offset: tuple = (5.0, 0.0, 0.0)
    # signal
    fc: float = 1e9
    bandwidth: float = 500e6
    pulse_T: float = 1e-6
    fs: float = 1.2e9
    n_samples: int = 4096
    upsample: int = 4
    # scene content
    n_scatterers: int = 3
    amp_lo: float = 1.0
    amp_hi: float = 1.0
    snr_db: float = 20.0
    seed: int = SEED_BASE + 1
    # samples dtype the workload is specified in ("c128" | "c64")
    sample_dtype: str = "c128"

    @property
    def n1(self) -> float:
        return 1.0

    @property
    def n2(self) -> float:
        return math.sqrt(self.eps_r)

    @property
    def n_voxels(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def voxel_pulses(self) -> int:
        return self.n_voxels * self.n_pulses


def config_spec(cfg: int) -> SceneSpec:
    """Scene specs of the five benchmark configurations (3 reuses 2's scene)."""
    if cfg == 1:
        # 41x41x21 grid: X in [19.2, 20.8], Y in [-0.8, 0.8] (0.04 m), Z in [-5.8, -4.2] (0.08 m)
        return SceneSpec("cfg1-small", 41, 41, 21, 0.04, 0.08, seed=SEED_BASE + 1)
    if cfg in (2, 3):
        return SceneSpec("cfg2-medium", 161, 161, 81, 0.02, 0.02, dem_n=256, dem_d=0.25,
                         dem_kind="fbm", dem_sigma=0.3, dem_beta=2.0, eps_r=6.0, n_pulses=1024,
                         bandwidth=800e6, fs=1.92e9, n_samples=8192, n_scatterers=50,
                         amp_lo=0.1, amp_hi=1.0, snr_db=15.0, seed=SEED_BASE + cfg)
    if cfg == 5:
        return SceneSpec("cfg5-large", 512, 512, 128, 0.02, 0.02, dem_n=1024, dem_d=0.125,
                         dem_kind="fbm", dem_sigma=0.5, dem_beta=2.2, eps_r=5.0, n_pulses=2048,
                         bandwidth=1e9, fs=2.4e9, n_samples=16384, n_scatterers=200,
                         amp_lo=0.1, amp_hi=1.0, snr_db=10.0, seed=SEED_BASE + 5,
                         sample_dtype="c64")
    raise ValueError(f"no scene spec for config {cfg}")


def scaled(spec: SceneSpec, **kw) -> SceneSpec:
    """A copy with fields replaced (smaller grids / fewer pulses for quick checks)."""
    return replace(spec, **kw)


# ------------------------------------------------------------------------------------
@dataclass
class Scene:
    spec: SceneSpec
    x_vec: np.ndarray
    y_vec: np.ndarray
    z: np.ndarray               # (ny_dem, nx_dem)
    tx: np.ndarray              # (Np, 3)
    rx: np.ndarray              # (Np, 3)
    gx: np.ndarray
    gy: np.ndarray
    gz: np.ndarray
    scat_pos: np.ndarray        # (S, 3)
    scat_amp: np.ndarray        # (S,)
    scat_voxel: np.ndarray      # (S, 3) grid indices (ix, iy, iz)
    raw: np.ndarray | None = None         # (Np, Ns) complex128 raw echoes
    chirp: np.ndarray | None = None
    reference: np.ndarray | None = None   # (Ns,) fftshifted matched-filter reference
    extra: dict = field(default_factory=dict)

    @property
    def lam(self) -> float:
        return C_LIGHT / self.spec.fc

    @property
    def fs_eff(self) -> float:
        return self.spec.fs * self.spec.upsample


def _streams(seed: int):
    ss = np.random.SeedSequence(seed)
    dem, scat, noise, extra = ss.spawn(4)
    return (np.random.Generator(np.random.PCG64(dem)), np.random.Generator(np.random.PCG64(scat)),
            np.random.Generator(np.random.PCG64(noise)), np.random.Generator(np.random.PCG64(extra)))


def grid_axes(spec: SceneSpec):
    cx, cy, cz = spec.center
    gx = cx + (np.arange(spec.nx) - (spec.nx - 1) / 2.0) * spec.dxy
    gy = cy + (np.arange(spec.ny) - (spec.ny - 1) / 2.0) * spec.dxy
    gz = cz + (np.arange(spec.nz) - (spec.nz - 1) / 2.0) * spec.dz
    return gx, gy, gz


def make_dem(spec: SceneSpec, rng: np.random.Generator):
    n, d = spec.dem_n, spec.dem_d
    cx, cy, _ = spec.center
    x_vec = cx + (np.arange(n) - (n - 1) / 2.0) * d
    y_vec = cy + (np.arange(n) - (n - 1) / 2.0) * d
    if spec.dem_kind == "plane":
        z = rng.normal(0.0, spec.dem_sigma, size=(n, n))
    else:
        kx = np.fft.fftfreq(n)
        k = np.sqrt(kx[None, :] ** 2 + kx[:, None] ** 2)
        k[0, 0] = 1.0
        amp = k ** (-spec.dem_beta / 2.0)
        amp[0, 0] = 0.0
        phase = rng.uniform(0.0, 2.0 * np.pi, size=(n, n))
        white = rng.normal(size=(n, n))
        H = amp * white * np.exp(1j * phase)
        z = np.real(np.fft.ifft2(H))
        z = z - z.mean()
        s = z.std()
        z = z * (spec.dem_sigma / s) if s > 0 else z
    return x_vec, y_vec, np.ascontiguousarray(z)


def make_trajectories(spec: SceneSpec):
    n = spec.n_pulses
    s = np.arange(n) / max(n - 1, 1)
    r = spec.r_max * (1.0 - s)
    th = 2.0 * np.pi * spec.turns * s
    tx = np.stack([r * np.cos(th), r * np.sin(th), np.full(n, spec.altitude)], axis=1)
    rx = tx + np.asarray(spec.rx_offset, dtype=np.float64)[None, :]
    return np.ascontiguousarray(tx), np.ascontiguousarray(rx)


def make_scatterers(spec: SceneSpec, rng: np.random.Generator, gx, gy, gz):
    S = spec.n_scatterers
    ix = rng.integers(2, spec.nx - 2, size=S) if spec.nx > 4 else rng.integers(0, spec.nx, size=S)
    iy = rng.integers(2, spec.ny - 2, size=S) if spec.ny > 4 else rng.integers(0, spec.ny, size=S)
    iz = rng.integers(1, spec.nz - 1, size=S) if spec.nz > 2 else rng.integers(0, spec.nz, size=S)
    pos = np.stack([gx[ix], gy[iy], gz[iz]], axis=1)
    if spec.amp_lo == spec.amp_hi:
        amp = np.full(S, spec.amp_lo)
    else:
        amp = np.exp(rng.uniform(np.log(spec.amp_lo), np.log(spec.amp_hi), size=S))
    return pos, amp, np.stack([ix, iy, iz], axis=1)


# ------------------------------------------------------------------------------------
# Vectorised FP64 Newton Fermat solve used for echo synthesis.  Same steps as the
# product's Newton kernels: flat-interface Snell start, node scan of +-W DEM nodes,
# active-set projected Newton on the 4 facets around the best node, one final step.
FLAT_ITERS = 4
POLISH_ITERS = 3


def search_nodes_for(x_vec, y_vec, radius_m: float = 1.5) -> int:
    """Node-scan half width W covering radius_m on the DEM's finer axis."""
    d = min((x_vec[-1] - x_vec[0]) / (len(x_vec) - 1), (y_vec[-1] - y_vec[0]) / (len(y_vec) - 1))
    return max(1, int(math.ceil(radius_m / d - 1e-9)))


def _elev(x_vec, y_vec, z, x, y):
    """Bilinear height with the nearest-edge value outside the DEM."""
    n, m = len(x_vec), len(y_vec)
    i = np.clip(np.searchsorted(x_vec, x, side="right") - 1, 0, n - 2)
    j = np.clip(np.searchsorted(y_vec, y, side="right") - 1, 0, m - 2)
    u = np.clip((x - x_vec[i]) / (x_vec[i + 1] - x_vec[i]), 0.0, 1.0)
    v = np.clip((y - y_vec[j]) / (y_vec[j + 1] - y_vec[j]), 0.0, 1.0)
    return (z[j, i] * (1 - u) * (1 - v) + z[j, i + 1] * u * (1 - v) + z[j + 1, i] * (1 - u) * v
            + z[j + 1, i + 1] * u * v)


def _facet_step(F, A, B, na, nb, u, v):
    x0, y0, dx, dy, z00, b, c, e = F
    x = x0 + u * dx
    y = y0 + v * dy
    h = z00 + b * u + c * v + e * u * v
    zx = (b + e * v) / dx
    zy = (c + e * u) / dy
    zxy = e / (dx * dy)
    r1x, r1y, r1z = x - A[:, 0], y - A[:, 1], h - A[:, 2]
    r2x, r2y, r2z = x - B[:, 0], y - B[:, 1], h - B[:, 2]
    q1 = r1x * r1x + r1y * r1y + r1z * r1z
    q2 = r2x * r2x + r2y * r2y + r2z * r2z
    g1 = na / np.sqrt(q1)
    g2 = nb / np.sqrt(q2)
    a1x, a1y = r1x + r1z * zx, r1y + r1z * zy
    a2x, a2y = r2x + r2z * zx, r2y + r2z * zy
    gx = g1 * a1x + g2 * a2x
    gy = g1 * a1y + g2 * a2y
    txx, tyy, txy = 1 + zx * zx, 1 + zy * zy, zx * zy
    hxx = g1 * (txx - a1x * a1x / q1) + g2 * (txx - a2x * a2x / q2)
    hyy = g1 * (tyy - a1y * a1y / q1) + g2 * (tyy - a2y * a2y / q2)
    hxy = g1 * (txy - a1x * a1y / q1) + g2 * (txy - a2x * a2y / q2) + (g1 * r1z + g2 * r2z) * zxy
    au = ((u <= 0) & (gx > 0)) | ((u >= 1) & (gx < 0))
    av = ((v <= 0) & (gy > 0)) | ((v >= 1) & (gy < 0))
    gs = g1 + g2
    det = hxx * hyy - hxy * hxy
    good = (det > 0) & (hxx > 0)
    dets = np.where(good, det, 1.0)
    su = np.where(good, -(hyy * gx - hxy * gy) / dets, -gx / gs)
    sv = np.where(good, -(hxx * gy - hxy * gx) / dets, -gy / gs)
    su1 = np.where(hxx > 0, -gx / np.where(hxx > 0, hxx, 1.0), -gx / gs)
    sv1 = np.where(hyy > 0, -gy / np.where(hyy > 0, hyy, 1.0), -gy / gs)
    su = np.where(au, 0.0, np.where(av, su1, su))
    sv = np.where(av, 0.0, np.where(au, sv1, sv))
    corner = au & av
    u = np.where(corner, u, np.clip(u + su / dx, 0.0, 1.0))
    v = np.where(corner, v, np.clip(v + sv / dy, 0.0, 1.0))
    return u, v


def _facet_eval(F, A, B, na, nb, u, v):
    x0, y0, dx, dy, z00, b, c, e = F
    X = np.stack([x0 + u * dx, y0 + v * dy, z00 + b * u + c * v + e * u * v], axis=1)
    return X, na * np.linalg.norm(X - A, axis=1) + nb * np.linalg.norm(X - B, axis=1)


def _facets(x_vec, y_vec, z, fi, fj):
    x0, y0 = x_vec[fi], y_vec[fj]
    z00, z01, z10, z11 = z[fj, fi], z[fj, fi + 1], z[fj + 1, fi], z[fj + 1, fi + 1]
    return (x0, y0, x_vec[fi + 1] - x0, y_vec[fj + 1] - y0, z00, z01 - z00, z10 - z00,
            z11 - z01 - z10 + z00)


def fermat_newton(x_vec, y_vec, z, A, B, na, nb, search_nodes=None):
    """Crossing points X minimising na|X-A| + nb|X-B| on the DEM surface (vectorised)."""
    A = np.asarray(A, dtype=np.float64)
    B = np.asarray(B, dtype=np.float64)
    W = search_nodes_for(x_vec, y_vec) if search_nodes is None else int(search_nodes)
    nxd, nyd = len(x_vec), len(y_vec)
    lower_b = nb >= na
    U, L, nu, nl = (A, B, na, nb) if lower_b else (B, A, nb, na)
    h0 = _elev(x_vec, y_vec, z, L[:, 0], L[:, 1])
    hx_, hy_ = L[:, 0] - U[:, 0], L[:, 1] - U[:, 1]
    D = np.sqrt(hx_ * hx_ + hy_ * hy_)
    ha, hb = np.abs(U[:, 2] - h0), np.abs(L[:, 2] - h0)
    s = np.clip(D * ha / (ha + hb + 1e-30), 0.0, D)
    for _ in range(FLAT_ITERS):
        q1 = np.sqrt(s * s + ha * ha)
        r = D - s
        q2 = np.sqrt(r * r + hb * hb)
        g = nu * s / q1 - nl * r / q2
        gp = nu * ha * ha / q1 ** 3 + nl * hb * hb / q2 ** 3
        s = np.clip(s - np.where(gp > 0, g / np.where(gp > 0, gp, 1.0), 0.0), 0.0, D)
    Dsafe = np.where(D >= 1e-9, D, 1.0)
    sx = np.where(D >= 1e-9, U[:, 0] + hx_ * (s / Dsafe), L[:, 0])
    sy = np.where(D >= 1e-9, U[:, 1] + hy_ * (s / Dsafe), L[:, 1])
    stepx = (x_vec[-1] - x_vec[0]) / (nxd - 1)
    stepy = (y_vec[-1] - y_vec[0]) / (nyd - 1)
    i_s = np.clip(np.floor((sx - x_vec[0]) / stepx + 0.5), 0, nxd - 1).astype(np.int64)
    j_s = np.clip(np.floor((sy - y_vec[0]) / stepy + 0.5), 0, nyd - 1).astype(np.int64)
    bestL = np.full(len(A), np.inf)
    bi, bj = i_s.copy(), j_s.copy()
    for di in range(-W, W + 1):
        ii = i_s + di
        okx = (ii >= 0) & (ii < nxd)
        iic = np.clip(ii, 0, nxd - 1)
        for dj in range(-W, W + 1):
            jj = j_s + dj
            ok = okx & (jj >= 0) & (jj < nyd)
            jjc = np.clip(jj, 0, nyd - 1)
            X = np.stack([x_vec[iic], y_vec[jjc], z[jjc, iic]], axis=1)
            Lv = na * np.linalg.norm(X - A, axis=1) + nb * np.linalg.norm(X - B, axis=1)
            m = ok & (Lv < bestL)
            bestL = np.where(m, Lv, bestL)
            bi = np.where(m, iic, bi)
            bj = np.where(m, jjc, bj)
    bfi = np.minimum(bi, nxd - 2)
    bfj = np.minimum(bj, nyd - 2)
    bestF = np.full(len(A), np.inf)
    bu = (bi - bfi).astype(np.float64)
    bv = (bj - bfj).astype(np.float64)
    for k in range(4):
        fi = bi - 1 + (k >> 1)
        fj = bj - 1 + (k & 1)
        ok = (fi >= 0) & (fj >= 0) & (fi <= nxd - 2) & (fj <= nyd - 2)
        fic, fjc = np.clip(fi, 0, nxd - 2), np.clip(fj, 0, nyd - 2)
        F = _facets(x_vec, y_vec, z, fic, fjc)
        u = (bi - fic).astype(np.float64)
        v = (bj - fjc).astype(np.float64)
        for _ in range(POLISH_ITERS):
            u, v = _facet_step(F, A, B, na, nb, u, v)
        _, Lf = _facet_eval(F, A, B, na, nb, u, v)
        m = ok & (Lf < bestF)
        bestF = np.where(m, Lf, bestF)
        bu, bv = np.where(m, u, bu), np.where(m, v, bv)
        bfi, bfj = np.where(m, fic, bfi), np.where(m, fjc, bfj)
    F = _facets(x_vec, y_vec, z, bfi, bfj)
    bu, bv = _facet_step(F, A, B, na, nb, bu, bv)
    X, _ = _facet_eval(F, A, B, na, nb, bu, bv)
    return X


def optical_paths(scene: Scene, points):
    """Per-pulse two-way optical path (Np, S) for the given target points (S, 3)."""
    sp = scene.spec
    Np = len(scene.tx)
    S = len(points)
    A = np.repeat(scene.tx, S, axis=0)                       # (Np*S, 3)
    Pm = np.tile(points, (Np, 1))
    Rm = np.repeat(scene.rx, S, axis=0)
    ida = fermat_newton(scene.x_vec, scene.y_vec, scene.z, A, Pm, sp.n1, sp.n2)
    volta = fermat_newton(scene.x_vec, scene.y_vec, scene.z, Pm, Rm, sp.n2, sp.n1)
    r1t = np.linalg.norm(A - ida, axis=1)
    r2t = np.linalg.norm(Pm - ida, axis=1)
    r1r = np.linalg.norm(Rm - volta, axis=1)
    r2r = np.linalg.norm(Pm - volta, axis=1)
    L = sp.n1 * r1t + sp.n2 * r2t + sp.n2 * r2r + sp.n1 * r1r
    return L.reshape(Np, S)


# ------------------------------------------------------------------------------------
def chirp_params(spec: SceneSpec):
    f0, f1 = -spec.bandwidth / 2.0, spec.bandwidth / 2.0
    nc = int(spec.pulse_T * spec.fs) + 1            # src/raw_data_processing.cpp:271
    return f0, f1, nc


def make_chirp(spec: SceneSpec):
    """LFM chirp exp(j 2 pi (f0 t + k/2 t^2)), t = n / fs (src/raw_data_processing.cpp:257-290)."""
    f0, f1, nc = chirp_params(spec)
    k = (f1 - f0) / spec.pulse_T
    t = np.arange(nc) / spec.fs
    ph = 2.0 * np.pi * (f0 * t + (k / 2.0) * t * t)
    return np.cos(ph) + 1j * np.sin(ph)


def matched_reference(chirp: np.ndarray, n: int) -> np.ndarray:
    """[second half of chirp, zeros, first half] (src/raw_data_processing.cpp:371-394)."""
    nc = len(chirp)
    half = nc // 2
    ref = np.zeros(n, dtype=np.complex128)
    ref[: nc - half] = chirp[half:]
    ref[n - half:] = chirp[:half]
    return ref


def synthesize_raw(scene: Scene, L: np.ndarray, rng: np.random.Generator, chunk: int = 64):
    """Raw echoes (Np, Ns) from optical paths L (Np, S)."""
    sp = scene.spec
    f0, f1, nc = chirp_params(sp)
    k = (f1 - f0) / sp.pulse_T
    half = nc // 2
    Np, S = L.shape
    raw = np.zeros((Np, sp.n_samples), dtype=np.complex128)
    tau = L / C_LIGHT
    carrier = scene.scat_amp[None, :] * np.exp(-2j * np.pi * sp.fc * tau)    # (Np, S)
    n_all = np.arange(sp.n_samples)
    for p0 in range(0, Np, chunk):
        p1 = min(Np, p0 + chunk)
        for s in range(S):
            c0 = tau[p0:p1, s] * sp.fs                        # echo centre in samples
            lo = np.maximum(np.floor(c0 - half).astype(np.int64), 0)
            hi = np.minimum(np.ceil(c0 + (nc - 1 - half)).astype(np.int64) + 1, sp.n_samples)
            for q in range(p1 - p0):
                if hi[q] <= lo[q]:
                    continue
                n = n_all[lo[q]:hi[q]]
                t = n / sp.fs - tau[p0 + q, s] + half / sp.fs      # time inside the chirp
                m = (t >= 0.0) & (t <= (nc - 1) / sp.fs)
                ph = 2.0 * np.pi * (f0 * t + (k / 2.0) * t * t)
                raw[p0 + q, lo[q]:hi[q]] += np.where(m, carrier[p0 + q, s] * np.exp(1j * ph), 0.0)
    if np.isfinite(sp.snr_db):
        sigma2 = nc / (10.0 ** (sp.snr_db / 10.0))
        noise = rng.normal(size=raw.shape) + 1j * rng.normal(size=raw.shape)
        raw += noise * math.sqrt(sigma2 / 2.0)
    return raw


def make_scene(spec: SceneSpec, with_raw: bool = True) -> Scene:
    rng_dem, rng_scat, rng_noise, _ = _streams(spec.seed)
    x_vec, y_vec, z = make_dem(spec, rng_dem)
    tx, rx = make_trajectories(spec)
    gx, gy, gz = grid_axes(spec)
    pos, amp, vox = make_scatterers(spec, rng_scat, gx, gy, gz)
    sc = Scene(spec, x_vec, y_vec, z, tx, rx, gx, gy, gz, pos, amp, vox)
    sc.chirp = make_chirp(spec)
    sc.reference = matched_reference(sc.chirp, spec.n_samples)
    if with_raw:
        L = optical_paths(sc, pos)
        sc.raw = synthesize_raw(sc, L, rng_noise)
    return sc


def pulse_compress_np(raw: np.ndarray, reference: np.ndarray) -> np.ndarray:
    """numpy pulse compression ifft(fft(raw) * conj(fft(ref))) per pulse (a cross-check)."""
    return np.fft.ifft(np.fft.fft(raw, axis=1) * np.conj(np.fft.fft(reference))[None, :], axis=1)


# ------------------------------------------------------------------------------------
# Served mixed workload: image-formation requests of different sizes over a few
# resident DEMs, arriving as a Poisson stream.
@dataclass
class ServeMix:
    dems: list                  # [(x_vec, y_vec, z, eps_r, sigma)]
    requests: list              # [Scene] (raw echoes not generated: synthesised on the device)
    dem_index: np.ndarray       # DEM of each request


def serve_mix(n_requests: int = 512, seed: int = SEED_BASE + 4, n_dems: int = 8, side=(21, 161),
              pulses=(128, 2048), samples_log2=(11, 14), scatterers=(5, 50), sigma=(0.1, 0.5),
              eps_r=(3.0, 9.0)) -> ServeMix:
    """Seeded request list of the served workload.

    Per request: grid side log-uniform over `side` (x = y = side, z = ceil(side / 2), 0.02 m
    voxels centred 20 m downrange and 5 m deep), pulse count log-uniform over `pulses`,
    fast-time samples 2^k with k uniform over `samples_log2` (log-uniform over powers of
    two), scatterer count uniform over `scatterers`, one of `n_dems` fBm DEMs (256 x 256
    at 0.25 m, beta 2, sigma uniform over `sigma`, eps_r uniform over `eps_r`).  Signal as
    the medium scene: f_c 1 GHz, B 800 MHz, fs 1.92 GHz, 1 us chirp, 15 dB SNR."""
    s_dem, s_req = np.random.SeedSequence(seed).spawn(2)
    rng_d = np.random.Generator(np.random.PCG64(s_dem))
    rng = np.random.Generator(np.random.PCG64(s_req))
    base = config_spec(2)
    dems = []
    for k in range(n_dems):
        sg = float(rng_d.uniform(*sigma))
        er = float(rng_d.uniform(*eps_r))
        dspec = replace(base, name=f"serve-dem{k}", dem_sigma=sg, eps_r=er)
        x_vec, y_vec, z = make_dem(dspec, rng_d)
        dems.append((x_vec, y_vec, z, er, sg))
    reqs, dem_idx = [], []
    for i in range(n_requests):
        sd = int(round(math.exp(rng.uniform(math.log(side[0]), math.log(side[1])))))
        npl = int(round(math.exp(rng.uniform(math.log(pulses[0]), math.log(pulses[1])))))
        ns = 1 << int(rng.integers(samples_log2[0], samples_log2[1] + 1))
        nsc = int(rng.integers(scatterers[0], scatterers[1] + 1))
        k = int(rng.integers(0, n_dems))
        rseed = int(rng.integers(0, 2**62))
        x_vec, y_vec, z, er, sg = dems[k]
        spec = replace(base, name=f"serve-req{i}", nx=sd, ny=sd, nz=(sd + 1) // 2, dem_sigma=sg, eps_r=er,
                       n_pulses=npl, n_samples=ns, n_scatterers=nsc, seed=rseed)
        _, rng_scat, _, _ = _streams(rseed)
        tx, rx = make_trajectories(spec)
        gx, gy, gz = grid_axes(spec)
        pos, amp, vox = make_scatterers(spec, rng_scat, gx, gy, gz)
        sc = Scene(spec, x_vec, y_vec, z, tx, rx, gx, gy, gz, pos, amp, vox)
        reqs.append(sc)
        dem_idx.append(k)
    return ServeMix(dems, reqs, np.asarray(dem_idx))


def poisson_arrivals(n: int, rate_per_s: float, seed: int = SEED_BASE + 40) -> np.ndarray:
    """Arrival times (s) of a Poisson stream: cumulative exponential gaps, first at 0."""
    rng = np.random.Generator(np.random.PCG64(seed))
    gaps = rng.exponential(1.0 / rate_per_s, size=n)
    gaps[0] = 0.0
    return np.cumsum(gaps)
