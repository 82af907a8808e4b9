"""Benchmark: bistatic SAR back-projection, voxel-pulses per second (Fermat included).

Workload: the medium scene (161 x 161 x 81 voxels at 0.02 m centred 20 m downrange and
5 m deep, 1024 pulses, 8192 fast-time samples x4 upsampled, 256 x 256 fBm DEM at
0.25 m with sigma 0.3 m, eps_r 6, 50 scatterers, 15 dB SNR; seeded synthetic data).

One step = the whole hot path on one batch: pulse compression + x4 upsampling of all
pulses (one launch) and the back-projection of every voxel with both Fermat solves of
every pulse (one launch), image left in HBM.

  value   mixed form (FP32 Newton scan/polish + FP64 final step, FP32 differential
          delays, complex64 samples, Kahan sums) with the raw pulses resident in HBM
  e2e     the same through the C ABI with host buffers: scene upload from pinned host
          memory, compression, back-projection and the image read back every step
  forms   the plain FP64 Newton form (the >= 2x comparator), the FP16-sample mixed form,
          and the reference's own algorithm (grid search, mean legs) in FP64 on the GPU
          over a voxel subset, with the accuracy of the mixed image against FP64

  serving the served mixed workload: 512 image-formation requests (grid side 21-161,
          128-2048 pulses, 2048-16384 samples, 8 resident fBm DEMs, 5-50 scatterers)
          through the continuous-batching server (bsar_server_*), arriving as a Poisson
          stream at 80 % of the capacity measured on a closed burst of the whole mix (the
          same 512 requests; a burst of only the first 64 measured 29 % more, and those
          carry 18 % less echo-synthesis work per voxel-pulse than the whole mix);
          latency p50 / p99 from submission to image on the host, echoes synthesised on
          the device at admission; beside it a sample of the same requests run serially
          in the plain FP64 form

--impl reference times the reference's CPU implementation (its own sources compiled
under oracle/_ref, OpenMP over the host cores) on a bounded voxel sample of the same
scene.  Multi-GPU (torchrun): every rank images its own z-slab of the same size (weak
scaling, no collective in the data path); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "c-_bistatic_sar_b200"))

METRIC = "BP voxel-pulses/s (Fermat incl.), mixed vs FP64 @<=1e-3 rel-L2; served p99 ms"
# DRAM bytes (read + write) of one k_bp_mixed launch on the full medium scene: a one-pass
# ncu capture of dram__bytes_read.sum + dram__bytes_write.sum of the headline command
# (4.06 MB + 2.47 MB; the gathers hit L2, and the image leaves L2 after the kernel ends)
TRAFFIC_BYTES = {2: 6.53e6}
UNIT = "voxel-pulses/s"


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None
        self.thread = None
        self.first = threading.Event()

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi's start-up (NVML initialisation) is kept out of the caller's
            # timed region: wait for the first sample
            self.first.wait(timeout=10)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])
            self.first.set()
        self.first.set()

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows if len(r) >= 9 for k in range(4)
                          if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm)}


# ------------------------------------------------------------------------------------
def l2_copy_gbs(torch, stream, mib: int = 32, reps: int = 50) -> float:
    """L2 bandwidth of this GPU, measured: a device copy between two buffers of `mib` MiB
    (both resident in the 126 MB L2 after the first pass), read + write bytes over the
    CUDA-event time of `reps` back-to-back copies, best of 5."""
    n = mib * (1 << 20) // 4
    a = torch.ones(n, dtype=torch.float32, device="cuda")
    b = torch.empty_like(a)
    best = 0.0
    with torch.cuda.stream(stream):
        for _ in range(3):
            b.copy_(a)
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                b.copy_(a)
            e1.record(stream)
            e1.synchronize()
            best = max(best, 2 * a.numel() * 4 * reps / (e0.elapsed_time(e1) / 1e3) / 1e9)
    del a, b
    return best


def fp32_flops_per_voxel_pulse(W: int) -> int:
    """Algorithmic FP32 work of the mixed kernel per voxel-pulse (FMA = 2 flops), counted
    from k_mixed.cu: per Fermat solve a (2W+1)^2 node scan at 17 flops per node, 4 facets x
    3 polish steps at 80 flops and 4 facet evaluations at 25, a 4-step flat start at 19
    flops (+ 20 setup); two solves per voxel-pulse plus 40 flops of delay / phase /
    interpolation / Kahan work."""
    per_solve = (2 * W + 1) ** 2 * 17 + 4 * 3 * 80 + 4 * 25 + 4 * 19 + 20
    return 2 * per_solve + 40


def sfu_ops_per_voxel_pulse(W: int) -> int:
    """MUFU operations per voxel-pulse: 2 rsqrt per scanned node, 4 per polish step
    (2 rsqrt + 2 rcp), 2 per facet evaluation, 2 per flat step; sincos = 2."""
    per_solve = (2 * W + 1) ** 2 * 2 + 4 * 3 * 4 + 4 * 2 + 4 * 2
    return 2 * per_solve + 2


def make_workload(cfg: int, rank: int, nz: int = 0):
    from bsar import scene as S

    spec = S.config_spec(cfg)
    if nz:
        spec = S.scaled(spec, nz=nz)
    # the large scene's echoes are synthesised on the GPU (bsar_scene_synthesize)
    sc = S.make_scene(spec, with_raw=spec.n_pulses * spec.n_samples <= (1 << 24))
    if rank:
        # weak scaling: rank r images the next z-slab of the same size
        sc.gz = sc.gz - rank * spec.nz * spec.dz
    return sc


def time_compress(ctx, torch, stream, sid, precision, reps=10):
    """Median device time of one scene compression (pulse compression + x4 upsampling into
    the form's storage), `reps` launches back to back after one untimed launch.  The raw
    pulses and the upsampled storage are larger than L2, so no flush is needed."""
    ctx.scene_compress(sid, precision)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for a, b in ev:
        a.record(stream)
        ctx.scene_compress(sid, precision)
        b.record(stream)
    torch.cuda.synchronize()
    return statistics.median(a.elapsed_time(b) for a, b in ev)


def time_device(ctx, torch, stream, sid, sc, precision, solver, legs, steps, warmup, gx=None, gy=None, gz=None):
    """Device time of `steps` steps (compression + back-projection), CUDA events on the
    library's stream; also the back-projection kernel alone."""
    gx = sc.gx if gx is None else gx
    gy = sc.gy if gy is None else gy
    gz = sc.gz if gz is None else gz
    nv = len(gx) * len(gy) * len(gz)
    img = torch.empty((nv, 2), dtype=torch.float64, device="cuda")
    ptr = img.data_ptr()

    def step(ev=None):
        if ev is not None:
            ev[2].record(stream)
        ctx.scene_compress(sid, precision)
        if ev is not None:
            ev[0].record(stream)
        ctx.backproject_device(sid, gx, gy, gz, ptr, solver=solver, legs=legs, precision=precision)
        if ev is not None:
            ev[1].record(stream)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    kev = [tuple(torch.cuda.Event(enable_timing=True) for _ in range(3)) for _ in range(steps)]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    launches0 = ctx.launches
    t0.record(stream)
    for k in range(steps):
        step(kev[k])
    t1.record(stream)
    torch.cuda.synchronize()
    total_ms = t0.elapsed_time(t1)
    bp_ms = [a.elapsed_time(b) for a, b, _ in kev]
    time_device.pc_ms = [c.elapsed_time(a) for a, b, c in kev]
    return total_ms, bp_ms, img, ctx.launches - launches0


def cpu_reference_rate(sc, seconds: float, threads: int, use_ref: bool = True, voxels=None, what=None):
    """Reference CPU path (grid search, mean legs) on a bounded voxel sample: `voxels`
    (flat indices in the reference's voxel order) when given, else random voxels of the
    grid, as many as take about `seconds`.  Returns (voxel-pulses/s for a full image,
    details incl. the sampled voxels, their values and the upsampled pulses)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    kind = "reference" if (use_ref and O.Reference.available()) else "port"
    impl = O.Reference() if kind == "reference" else O.Oracle()
    sp = sc.spec
    dem = O.Dem(sc.x_vec, sc.y_vec, sc.z)
    # pulse compression + upsampling of every pulse (processRawData / splineInterpolation)
    t = time.perf_counter()
    rc = impl.fft_correlate(sc.raw, sc.reference)
    t_pc = time.perf_counter() - t
    t = time.perf_counter()
    rc = impl.spline_upsample(rc, sp.upsample)
    t_up = time.perf_counter() - t
    nv_total = sp.nx * sp.ny * sp.nz
    rng = np.random.default_rng(0x5A4B0002)
    kw = dict(legs="mean")
    if kind == "reference":
        kw["nthreads"] = threads
    else:
        kw["solver"] = "grid"

    last = {}

    def run(vox):
        t0 = time.perf_counter()
        vals = impl.backproject(dem, sc.tx, sc.rx, rc, sc.gx, sc.gy, sc.gz, sp.n1, sp.n2, 3e8, sc.fs_eff, sc.lam,
                                voxels=vox, **kw)
        last["vox"], last["vals"] = vox, vals
        return time.perf_counter() - t0

    if voxels is not None:
        n1 = len(voxels)
        dt1 = run(np.asarray(voxels, dtype=np.int64))
        what = what or f"{n1} listed voxels"
    else:
        n0 = max(threads, 1)
        dt0 = run(rng.choice(nv_total, size=n0, replace=False))
        n1 = max(n0, int(n0 * seconds / max(dt0, 1e-3)) // n0 * n0)
        dt1 = run(rng.choice(nv_total, size=n1, replace=False)) if n1 > n0 else dt0
        what = f"{n1} random voxels"
    per_voxel = dt1 / n1
    full_s = t_pc + t_up + per_voxel * nv_total
    rate = nv_total * sp.n_pulses / full_s
    return rate, {"kind": kind, "cores": threads, "sample": (
        f"{what} of the {sp.nx}x{sp.ny}x{sp.nz} grid x {sp.n_pulses} pulses (grid-search Fermat, "
        f"mean legs, as shipped) in {dt1:.1f} s + full pulse compression {t_pc:.1f} s and upsampling "
        f"{t_up:.1f} s; rate = full-image voxel-pulses / (compression + upsampling + per-voxel time x "
        f"{nv_total} voxels), extrapolated linearly in the voxel count"), "per_voxel_s": per_voxel, "pc_s": t_pc,
        "upsample_s": t_up, "voxels": last["vox"], "values": last["vals"], "rc": rc}


def parity_sample(sp, scat_voxel, seed: int, target: int = 3000):
    """Seeded parity sample of the imaging grid: a uniform sub-lattice (every s-th voxel on
    each axis from a random offset, s chosen for about `target` voxels) and the 3 x 3 x 3
    neighbourhood of every scatterer.  Returns the voxels' grid indices (n, 3) as (ix, iy, iz),
    the lattice's axis indices, the neighbourhoods' axis ranges and the neighbourhood each
    voxel belongs to (-1: lattice)."""
    rng = np.random.default_rng(seed)
    s = max(1, int(math.ceil((sp.n_voxels / target) ** (1.0 / 3.0))))
    while math.prod(-(-n // s) for n in (sp.nx, sp.ny, sp.nz)) > target:     # thin grids: widen the stride
        s += 1
    lat = [np.arange(rng.integers(0, min(s, n)), n, s) for n in (sp.nx, sp.ny, sp.nz)]
    ii = np.stack(np.meshgrid(*lat, indexing="ij"), axis=-1).reshape(-1, 3)
    groups = [np.full(len(ii), -1)]
    hoods = []
    for k, (x, y, z) in enumerate(np.asarray(scat_voxel)):
        ax = [np.arange(max(c - 1, 0), min(c + 2, n)) for c, n in ((x, sp.nx), (y, sp.ny), (z, sp.nz))]
        hoods.append(ax)
        h = np.stack(np.meshgrid(*ax, indexing="ij"), axis=-1).reshape(-1, 3)
        ii = np.concatenate([ii, h])
        groups.append(np.full(len(h), k))
    return ii, lat, hoods, np.concatenate(groups)


def flat_voxels(sp, ii):
    """Grid indices (ix, iy, iz) -> the reference's flat voxel order (z -> x -> y)."""
    return (ii[:, 2] * sp.nx + ii[:, 0]) * sp.ny + ii[:, 1]


def sample_stats(x, ref, groups):
    """Errors of sample values x against ref: rel-L2, max phase error over the voxels at or
    above 1e-3 of the largest magnitude, the sample's argmax, and per scatterer whether the
    argmax of its 3 x 3 x 3 neighbourhood is the same voxel."""
    m = np.abs(ref) >= 1e-3 * np.abs(ref).max()
    hood = [np.flatnonzero(groups == k) for k in range(int(groups.max()) + 1)]
    same = sum(int(np.argmax(np.abs(x[h])) == np.argmax(np.abs(ref[h]))) for h in hood if len(h))
    return {"rel_l2": float(np.linalg.norm(x - ref) / np.linalg.norm(ref)),
            "max_abs": float(np.abs(x - ref).max()),
            "max_phase_err_rad": float(np.abs(np.angle(x[m] * np.conj(ref[m]))).max()),
            "argmax_match": bool(np.argmax(np.abs(x)) == np.argmax(np.abs(ref))),
            "scatterer_argmax_match": f"{same}/{len(hood)}"}


def parity_block(ctx, sid, sc, ii, lat, hoods, groups, det, full_images, W):
    """Every form on the parity sample against the CPU: the GPU reference algorithm (grid
    search, mean legs, FP64) against the reference's own compiled code on the same voxels;
    the GPU FP64 Newton, mixed and mixed-FP16 images (the full-grid images of this run,
    read at the sample voxels) against the oracle's FP64 Newton on those voxels."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    sp = sc.spec
    # GPU reference algorithm on the sample: the lattice as one grid, each neighbourhood as
    # one 3 x 3 x 3 grid (a voxel's FP64 value does not depend on the grid around it)
    parts = [ctx.backproject(sid, sc.gx[lat[0]], sc.gy[lat[1]], sc.gz[lat[2]], solver="grid", legs="mean",
                             precision="fp64").reshape(-1)]
    for ax in hoods:
        parts.append(ctx.backproject(sid, sc.gx[ax[0]], sc.gy[ax[1]], sc.gz[ax[2]], solver="grid", legs="mean",
                                     precision="fp64").reshape(-1))
    gpu_grid = np.concatenate(parts)
    t = time.perf_counter()
    orc = O.Oracle().backproject(O.Dem(sc.x_vec, sc.y_vec, sc.z), sc.tx, sc.rx, det["rc"], sc.gx, sc.gy, sc.gz, sp.n1,
                                 sp.n2, 3e8, sc.fs_eff, sc.lam, legs="per_pulse", solver="newton",
                                 voxels=flat_voxels(sp, ii), search_nodes=W)
    t_orc = time.perf_counter() - t
    at = (ii[:, 0], ii[:, 1], ii[:, 2])
    return {"voxels": int(len(ii)),
            "sample": (f"uniform sub-lattice {len(lat[0])}x{len(lat[1])}x{len(lat[2])} (seeded offsets) + 3x3x3 around "
                       f"each of {len(hoods)} scatterers"),
            "fp64_grid_mean_vs_reference": sample_stats(gpu_grid, det["values"], groups),
            "fp64_newton_vs_oracle": sample_stats(full_images["fp64_newton"][at], orc, groups),
            "mixed_vs_oracle": sample_stats(full_images["mixed"][at], orc, groups),
            "mixed_fp16_vs_oracle": sample_stats(full_images["mixed_fp16"][at], orc, groups),
            "oracle_newton_cpu_s": t_orc,
            "bars": "FP64 forms rel-L2 <= 1e-9; mixed forms rel-L2 <= 1e-3, phase <= 0.01 rad; same argmax"}


def config5_leg(ctx, torch, stream, nz: int = 8, steps: int = 2, cpu_voxels: int = 180, hoods: int = 4):
    """The large scene (512 x 512 grid at 0.02 m, 2048 pulses, 16384 -> 65536 samples,
    1024^2 fBm DEM at 0.125 m, so 25 x 25 node scans) on a z-slab of `nz` slices: pulse
    compression + x4 upsampling and the mixed back-projection timed per step; the mixed
    image against the GPU FP64 Newton image on one z-slice; mixed crossing points against
    FP64; a CPU sample (uniform sub-lattice of the slab + the neighbourhoods of up to
    `hoods` scatterers inside it) run by the reference's compiled code against the GPU
    reference algorithm, and by the oracle's FP64 Newton against the GPU FP64 Newton and
    mixed values.  Echoes are synthesised on the GPU."""
    import bsar
    from bsar import scene as S

    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    spec = S.scaled(S.config_spec(5), nz=nz)
    sc = S.make_scene(spec, with_raw=False)
    s0 = bsar.synthesize_scene(ctx, sc)
    sc.raw = ctx.scene_read_samples(s0, spec.n_pulses, spec.n_samples)
    ctx.scene_release(s0)
    sid = bsar.upload_scene(ctx, sc)
    W = S.search_nodes_for(sc.x_vec, sc.y_vec)
    vp = spec.voxel_pulses
    total_ms, bp_ms, img_mixed, _ = time_device(ctx, torch, stream, sid, sc, "mixed", "newton", "per_pulse", steps, 1)
    pc_ms = [float(x) for x in time_device.pc_ms]
    mixed = img_mixed.cpu().numpy().view(np.complex128).reshape(spec.nx, spec.ny, spec.nz)
    del img_mixed
    # FP64 Newton on the first z-slice of the slab
    torch.cuda.synchronize()
    t = time.perf_counter()
    ref_slice = ctx.backproject(sid, sc.gx, sc.gy, sc.gz[:1], solver="newton", legs="per_pulse", precision="fp64")
    torch.cuda.synchronize()
    t64 = time.perf_counter() - t
    mx = mixed[:, :, :1]
    m = np.abs(ref_slice) >= 1e-3 * np.abs(ref_slice).max()
    acc = {"mixed_vs_fp64_newton_slice": {
        "voxels": int(ref_slice.size), "rel_l2": float(np.linalg.norm(mx - ref_slice) / np.linalg.norm(ref_slice)),
        "max_phase_err_rad": float(np.abs(np.angle(mx[m] * np.conj(ref_slice[m]))).max()),
        "argmax_match": bool(np.argmax(np.abs(mx)) == np.argmax(np.abs(ref_slice)))}}
    # crossing points: mixed vs FP64 on random (pulse, voxel) pairs of the slab
    rng = np.random.default_rng(0x5A4B0D5)
    pi = rng.integers(0, spec.n_pulses, 1 << 14)
    vi = rng.integers(0, [spec.nx, spec.ny, spec.nz], size=(1 << 14, 3))
    P = np.stack([sc.gx[vi[:, 0]], sc.gy[vi[:, 1]], sc.gz[vi[:, 2]]], axis=1)
    demA = bsar.DemArrays(sc.x_vec, sc.y_vec, sc.z)
    cross = dpath = 0.0
    for ant, na, nb, first in ((sc.tx, spec.n1, spec.n2, True), (sc.rx, spec.n2, spec.n1, False)):
        p1, p2 = (ant[pi], P) if first else (P, ant[pi])
        x64 = ctx.refraction_points(demA, p1, p2, na, nb, solver="newton")
        x32 = ctx.refraction_points(demA, p1, p2, na, nb, solver="newton", precision="mixed")
        cross = max(cross, float(np.linalg.norm(x32 - x64, axis=1).max()))
        path = lambda X: na * np.linalg.norm(p1 - X, axis=1) + nb * np.linalg.norm(p2 - X, axis=1)  # noqa: E731
        dpath = max(dpath, float(np.abs(path(x32) - path(x64)).max()))
    acc["mixed_fermat_crossing_max_err_m"] = cross
    acc["mixed_fermat_path_max_err_m"] = dpath
    acc["fermat_sample"] = "16384 random (pulse, voxel) pairs per leg"
    # CPU sample: the reference (grid search, mean legs) and the oracle's FP64 Newton
    inside = [k for k, v in enumerate(sc.scat_voxel) if 1 <= v[2] <= spec.nz - 2][:hoods]
    ii, lat, hd, groups = parity_sample(spec, sc.scat_voxel[inside], 0x5A4B0005, target=cpu_voxels)
    threads = os.cpu_count() or 1
    what = f"{len(ii)} sample voxels of the {spec.nz}-slice slab ({int((groups < 0).sum())} on a sub-lattice + " \
           f"the 3x3x3 neighbourhoods of {len(hd)} scatterers)"
    rate, det = cpu_reference_rate(sc, 0.0, threads, voxels=flat_voxels(spec, ii), what=what)
    parts = [ctx.backproject(sid, sc.gx[lat[0]], sc.gy[lat[1]], sc.gz[lat[2]], solver="grid", legs="mean",
                             precision="fp64").reshape(-1)]
    parts64 = [ctx.backproject(sid, sc.gx[lat[0]], sc.gy[lat[1]], sc.gz[lat[2]], solver="newton", legs="per_pulse",
                               precision="fp64").reshape(-1)]
    for ax in hd:
        parts.append(ctx.backproject(sid, sc.gx[ax[0]], sc.gy[ax[1]], sc.gz[ax[2]], solver="grid", legs="mean",
                                     precision="fp64").reshape(-1))
        parts64.append(ctx.backproject(sid, sc.gx[ax[0]], sc.gy[ax[1]], sc.gz[ax[2]], solver="newton",
                                       legs="per_pulse", precision="fp64").reshape(-1))
    orc = O.Oracle().backproject(O.Dem(sc.x_vec, sc.y_vec, sc.z), sc.tx, sc.rx, det["rc"], sc.gx, sc.gy, sc.gz,
                                 spec.n1, spec.n2, 3e8, sc.fs_eff, sc.lam, legs="per_pulse", solver="newton",
                                 voxels=flat_voxels(spec, ii), search_nodes=W)
    at = (ii[:, 0], ii[:, 1], ii[:, 2])
    acc["vs_cpu_sample"] = {
        "voxels": int(len(ii)),
        "fp64_grid_mean_vs_reference": sample_stats(np.concatenate(parts), det["values"], groups),
        "fp64_newton_vs_oracle": sample_stats(np.concatenate(parts64), orc, groups),
        "mixed_vs_oracle": sample_stats(mixed[at], orc, groups)}
    ctx.scene_release(sid)
    bp = statistics.mean(bp_ms)
    ns = spec.n_samples
    pc = statistics.median(pc_ms)
    pc_bytes = spec.n_pulses * (16 * ns + 8 * ns * spec.upsample)
    return {"workload": workload_name(spec) + f" (z-slab of {nz} slices)",
            "voxel_pulses_per_s": vp / (total_ms / steps / 1e3), "ms_per_step": total_ms / steps,
            "bp_kernel_ms": bp, "bp_voxel_pulses_per_s": vp / (bp / 1e3), "fermat_solves_per_s": 2 * vp / (bp / 1e3),
            "node_scan_half_width": W,
            "pulse_compression": {"ms": pc, "samples_per_s": spec.n_pulses * ns / (pc / 1e3),
                                  "achieved_gbs": pc_bytes / (pc / 1e3) / 1e9},
            "fp64_newton_slice_s": t64, "fp64_newton_voxel_pulses_per_s": ref_slice.size * spec.n_pulses / t64,
            "accuracy": acc,
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": det["cores"], "kind": det["kind"],
                             "sample": det["sample"]},
            "steps": steps}


def serve_leg(ctx, torch, n_requests: int, burst: int, fp64_sample: int, load: float = 0.8, tiles: int = 0):
    """Served mixed workload through bsar_server_* (see the module docstring)."""
    import bsar
    from bsar import scene as S

    mix = S.serve_mix(n_requests)
    reqs = mix.requests
    vp = np.array([r.spec.voxel_pulses for r in reqs], dtype=np.float64)
    dems = {}

    def submit(srv, i):
        r = reqs[i]
        if id(r.z) not in dems:
            dems[id(r.z)] = bsar.DemArrays(r.x_vec, r.y_vec, r.z)
        sp = r.spec
        return srv.submit(dems[id(r.z)], r.tx, r.rx, r.gx, r.gy, r.gz, n_samples=sp.n_samples, scat_pos=r.scat_pos,
                          scat_amp=r.scat_amp, snr_db=sp.snr_db, seed=sp.seed, upsample=sp.upsample, n1=sp.n1,
                          n2=sp.n2, c=3e8, fc=sp.fc, fs=sp.fs, chirp_f0=-sp.bandwidth / 2, chirp_f1=sp.bandwidth / 2,
                          chirp_T=sp.pulse_T, precision="mixed")

    budget = 120 * 10**9
    out = {"requests": n_requests, "hbm_budget_bytes": budget, "total_voxel_pulses": float(vp.sum()),
           "tiles_per_launch": tiles or "two waves of resident CTAs"}
    # closed burst: capacity of the server on this mix (burst <= 0: all of its requests)
    burst = n_requests if burst <= 0 else min(burst, n_requests)
    with bsar.Server(ctx, hbm_budget_bytes=budget, tiles_per_launch=tiles) as srv:
        submit(srv, 0)
        srv.wait(1)                                            # warm-up (graph capture, first admission)
        t = time.perf_counter()
        ids = [submit(srv, i) for i in range(burst)]
        for i in ids:
            srv.wait(i)
        dt = time.perf_counter() - t
    cap_vps = float(vp[:burst].sum()) / dt
    rate = load * cap_vps / float(vp.mean())                  # requests/s
    out["capacity"] = {"voxel_pulses_per_s": cap_vps, "requests": burst, "seconds": dt,
                       "requests_per_s": cap_vps / float(vp.mean())}
    # open loop: Poisson arrivals at `load` x capacity
    arrivals = S.poisson_arrivals(n_requests, rate)
    with ClockSampler(torch.cuda.current_device()) as clk:
        with bsar.Server(ctx, hbm_budget_bytes=budget, tiles_per_launch=tiles) as srv:
            submit(srv, 0)
            srv.wait(1)
            t0 = time.perf_counter()
            ids = []
            for i in range(n_requests):
                d = t0 + arrivals[i] - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                ids.append(submit(srv, i))
            lat = [srv.wait(i)[1] for i in ids]
            wall = time.perf_counter() - t0
            st = srv.stats()
    lat = np.asarray(lat)
    out["served"] = {"arrival_rate_per_s": rate, "load": load, "voxel_pulses_per_s": float(vp.sum()) / wall,
                     "seconds": wall, "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                     "mean_ms": float(lat.mean()), "max_ms": float(lat.max()), "launches": int(st["launches"]),
                     "tiles": int(st["tiles"]), "peak_inflight": int(st["peak_inflight"]),
                     "peak_reserved_gb": st["peak_reserved_bytes"] / 1e9, "failed": int(st["failed"]),
                     "batch_busy_fraction": st["batch_busy_s"] / wall}
    # a request cannot finish sooner than its own work at the full measured capacity
    floor_ms = np.sort(vp / cap_vps * 1e3)
    out["served"]["p99_service_floor_ms"] = float(np.percentile(floor_ms, 99))
    out["served"]["p50_service_floor_ms"] = float(np.percentile(floor_ms, 50))
    out["clocks"] = clk.summary()
    # the same requests one after another in the plain FP64 form (a spread sample)
    idx = np.linspace(0, n_requests - 1, min(fp64_sample, n_requests)).astype(int)
    t_fp64 = 0.0
    t_mixed = 0.0
    for i in idx:
        r = reqs[i]
        for form, acc in (("fp64", "t_fp64"), ("mixed", "t_mixed")):
            torch.cuda.synchronize()
            t = time.perf_counter()
            sid = bsar.synthesize_scene(ctx, r)
            ctx.backproject(sid, r.gx, r.gy, r.gz, solver="newton", legs="per_pulse", precision=form)
            ctx.scene_release(sid)
            dt = time.perf_counter() - t
            if form == "fp64":
                t_fp64 += dt
            else:
                t_mixed += dt
    vs = float(vp[idx].sum())
    out["serial_fp64"] = {"voxel_pulses_per_s": vs / t_fp64, "sample_requests": int(len(idx)),
                          "sample_voxel_pulses": vs, "seconds": t_fp64,
                          "est_total_seconds": t_fp64 * float(vp.sum()) / vs}
    out["serial_mixed"] = {"voxel_pulses_per_s": vs / t_mixed, "seconds": t_mixed}
    out["served_capacity_vs_serial_fp64"] = cap_vps / (vs / t_fp64)
    return out


def workload_name(sp) -> str:
    """The workload a bench line is quoted on (both arms name it the same way)."""
    return (f"{sp.name}: {sp.nx}x{sp.ny}x{sp.nz} voxels at {sp.dxy} m, {sp.n_pulses} pulses, "
            f"{sp.n_samples}->{sp.n_samples * sp.upsample} fast-time samples, "
            f"{sp.dem_n}^2 fBm DEM ({sp.dem_d} m, sigma {sp.dem_sigma} m), eps_r {sp.eps_r}, "
            f"{sp.n_scatterers} scatterers, {sp.snr_db} dB")


def kernel_tour():
    """One launch of every library kernel on moderate sizes: the profiling case behind the
    per-kernel summaries (inputs larger than L2 where a kernel streams memory)."""
    import tempfile

    import bsar
    from bsar import scene as S

    ctx = bsar.Context(0)
    tmp = tempfile.mkdtemp()
    # medium-scene signal and DEM on a 161 x 161 x 2 grid, 1024 pulses x 8192 samples
    sp = S.scaled(S.config_spec(2), nz=2)
    sc = S.make_scene(sp)
    dem = bsar.DemArrays(sc.x_vec, sc.y_vec, sc.z)
    sid = bsar.upload_scene(ctx, sc)
    ctx.scene_compress(sid, "mixed")          # k_ref_spectrum<float>, k_pulse_compress_rf<13>
    ctx.scene_compress(sid, "fp64")           # k_ref_spectrum<double>, k_pulse_compress<double>
    ctx.backproject(sid, sc.gx, sc.gy, sc.gz, solver="newton", legs="per_pulse", precision="mixed")  # k_ref_ranges, k_bp_mixed
    ctx.backproject(sid, sc.gx, sc.gy, sc.gz[:1], solver="newton", legs="per_pulse", precision="fp64")  # k_bp_plain<1,1>
    ctx.backproject(sid, sc.gx, sc.gy[:60], sc.gz[:1], solver="grid", legs="mean", precision="fp64")  # k_bp_plain<0,0>
    ctx.scene_release(sid)
    ctx.scene_release(bsar.synthesize_scene(ctx, sc))           # k_echo_paths, k_echo_synth
    # 16384-sample pulses in FP64: thread-block clusters (k_ref_spectrum_cl, k_pulse_compress_cl)
    sc5 = S.make_scene(S.scaled(S.config_spec(5), n_pulses=256, nx=16, ny=16, nz=2))
    s5 = bsar.upload_scene(ctx, sc5)
    ctx.scene_compress(s5, "fp64")
    ctx.scene_release(s5)
    # pulse files in the simulator's row-major layout (k_transpose_c128), real-valued (k_real_to_c128)
    raw = sc.raw[:256]
    common = dict(n1=sp.n1, n2=sp.n2, fc=sp.fc, fs=sp.fs, chirp_f0=-sp.bandwidth / 2, chirp_f1=sp.bandwidth / 2,
                  chirp_T=sp.pulse_T)
    p1 = os.path.join(tmp, "raw.bin")
    bsar.native.matrix_write(p1, np.ascontiguousarray(raw.T))
    ctx.scene_release(ctx.scene_upload_file(dem, sc.tx[:256], sc.rx[:256], p1, layout="row_major", kind="raw",
                                            **common))
    p2 = os.path.join(tmp, "real.bin")
    bsar.native.matrix_write(p2, np.ascontiguousarray(raw.real.T))
    s4 = ctx.scene_upload_file(dem, sc.tx[:256], sc.rx[:256], p2, layout="row_major", kind="compressed", **common)
    ctx.scene_compress(s4, "mixed")           # k_upsample_store
    ctx.scene_compress(s4, "fp64")            # k_spline
    ctx.scene_release(s4)
    ctx.fft(sc.raw[:512])                     # k_fft_rows
    rng = np.random.default_rng(3)
    n = 1 << 16
    P = np.stack([rng.uniform(19, 21, n), rng.uniform(-1.5, 1.5, n), rng.uniform(-6, -4, n)], 1)
    A = sc.tx[rng.integers(0, sp.n_pulses, n)]
    ctx.refraction_points(dem, A, P, sp.n1, sp.n2, solver="newton")                      # k_refraction_points<1>
    ctx.refraction_points(dem, A, P, sp.n1, sp.n2, solver="newton", precision="mixed")   # k_refraction_mixed
    ctx.dem_elevation(dem, P[:, :2])                                                      # k_dem_elevation
    ctx.close()
    print(json.dumps({"kernel_tour": "done"}), flush=True)
    return 0


def run_reference(args):
    """--impl reference: the reference's CPU implementation on the box's host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from bsar import scene as S

    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    sc = make_workload(args.config, 0, args.nz)
    if sc.raw is None:                     # no GPU on this arm: numpy echo synthesis
        sc = S.make_scene(sc.spec)
    sp = sc.spec
    rates = []
    details = None
    for k in range(args.warmup + args.steps):
        r, details = cpu_reference_rate(sc, args.ref_seconds, threads)
        if k >= args.warmup:
            rates.append(r)
    value = statistics.mean(rates)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sp.voxel_pulses / value * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded; no dataset)",
            "config": {"workload": workload_name(sp), "form": "reference CPU (grid search, mean legs)",
                       "parallelism": f"rank 0 only, {details['cores']} host threads"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": details["cores"], "kind": details["kind"],
                             "sample": details["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="bsar", choices=["bsar", "reference"])
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--ref-seconds", type=float, default=10.0, help="CPU work per reference sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the comparator forms")
    ap.add_argument("--nz", type=int, default=0, help="z-slices of the imaging grid (0: the scene's own; a "
                    "smaller grid of the same scene is the profiling case)")
    ap.add_argument("--serve-requests", type=int, default=512, help="requests of the served workload (0: skip)")
    ap.add_argument("--serve-burst", type=int, default=0,
                    help="requests of the capacity burst (0: the whole mix, the requests the open loop serves)")
    ap.add_argument("--serve-fp64-sample", type=int, default=24, help="requests run serially in FP64")
    ap.add_argument("--serve-only", action="store_true", help="only the served workload")
    ap.add_argument("--serve-tiles", type=int, default=0, help="work items per launch (0: two waves of CTAs)")
    ap.add_argument("--no-config5", action="store_true", help="skip the large-scene slab leg")
    ap.add_argument("--kernel-tour", action="store_true", help="launch every kernel once (profiling case) and exit")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.kernel_tour:
        return kernel_tour()

    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta

        dist_mod.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
        dist = dist_mod

    import bsar

    if args.serve_only:
        ctx = bsar.Context(local)
        res = serve_leg(ctx, torch, args.serve_requests, args.serve_burst, args.serve_fp64_sample,
                        tiles=args.serve_tiles)
        if rank == 0:
            print(json.dumps({"serving": res}), flush=True)
        ctx.close()
        return 0

    sc = make_workload(args.config, rank, args.nz)
    sp = sc.spec
    stream = torch.cuda.Stream()
    ctx = bsar.Context(local)
    ctx.set_stream(stream.cuda_stream)
    if sc.raw is None:
        s0 = bsar.synthesize_scene(ctx, sc)
        sc.raw = ctx.scene_read_samples(s0, sp.n_pulses, sp.n_samples)
        ctx.scene_release(s0)
    sid = bsar.upload_scene(ctx, sc)
    W = bsar.scene.search_nodes_for(sc.x_vec, sc.y_vec)
    nv = sp.n_voxels
    vp = nv * sp.n_pulses

    def barrier():
        if dist:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if not dist:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---------------- headline: mixed form, inputs resident in HBM -----------------
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        total_ms, bp_ms, img_mixed, launches = time_device(ctx, torch, stream, sid, sc, "mixed", "newton",
                                                           "per_pulse", args.steps, args.warmup)
    torch.cuda.synchronize()
    barrier()
    total_ms = max_over_ranks(total_ms)
    ms_per_step = total_ms / args.steps
    value = world * vp / (ms_per_step / 1e3)
    bp_avg_ms = max_over_ranks(statistics.mean(bp_ms))

    # ---------------- strong split (N > 1): one grid, z-slabs over the ranks -----------
    strong = None
    if dist:
        from bsar import shard

        gz_full = sc.gz + rank * sp.nz * sp.dz            # the grid rank 0 images in the weak mode
        barrier()
        torch.cuda.synchronize()
        t = time.perf_counter()
        full = shard.backproject_scene(ctx, sid, sc.gx, sc.gy, gz_full, dist, solver="newton", legs="per_pulse",
                                       precision="mixed")
        torch.cuda.synchronize()
        strong_s = max_over_ranks(time.perf_counter() - t)
        b, e = shard.z_slab(sp.nz, rank, world)
        strong = {"value": vp / strong_s, "unit": UNIT, "seconds": strong_s, "slab_z": [b, e],
                  "image_checksum": float(np.abs(full).sum()),
                  "note": "the medium grid once, z-slabs over the ranks (bsar.shard.backproject_scene), slabs "
                          "gathered over NCCL; wall clock max over ranks, host image included"}

    # ---------------- e2e through the C ABI with host buffers ----------------------
    raw_pinned = torch.empty(sc.raw.shape, dtype=torch.complex128, pin_memory=True)
    raw_pinned.numpy()[...] = sc.raw
    dem = bsar.DemArrays(sc.x_vec, sc.y_vec, sc.z)
    f0, f1 = -sp.bandwidth / 2, sp.bandwidth / 2
    # the image lands in pinned host memory
    img_pinned = torch.empty((sp.nx, sp.ny, sp.nz), dtype=torch.complex128, pin_memory=True)
    img_host = img_pinned.numpy()

    def e2e_step():
        s = ctx.scene_upload(dem, sc.tx, sc.rx, raw_pinned.numpy(), upsample=sp.upsample, n1=sp.n1, n2=sp.n2,
                             c=3e8, fc=sp.fc, fs=sp.fs, chirp_f0=f0, chirp_f1=f1, chirp_T=sp.pulse_T)
        out = ctx.backproject(s, sc.gx, sc.gy, sc.gz, solver="newton", legs="per_pulse", precision="mixed",
                              out=img_host)
        ctx.scene_release(s)
        return out

    e2e_steps = max(1, min(args.steps, 3))
    if args.warmup > 0:
        e2e_step()
    torch.cuda.synchronize()
    barrier()
    with ClockSampler(local) as clk_e2e:
        t = time.perf_counter()
        for _ in range(e2e_steps):
            img_host = e2e_step()
        torch.cuda.synchronize()
        e2e_s = max_over_ranks((time.perf_counter() - t) / e2e_steps)
    barrier()
    h2d = (sc.raw.nbytes + sc.tx.nbytes + sc.rx.nbytes + sc.x_vec.nbytes + sc.y_vec.nbytes + sc.z.nbytes
           + 8 * (len(sc.gx) + len(sc.gy) + len(sc.gz)))
    d2h = img_host.nbytes

    # ---------------- comparator forms + accuracy ----------------------------------
    forms = {}
    acc = {}
    full_images = None
    if not args.no_forms:
        fs = max(1, min(2, args.steps))
        t64, bp64, img64, _ = time_device(ctx, torch, stream, sid, sc, "fp64", "newton", "per_pulse", fs, 1)
        forms["fp64_newton"] = {"value": world * vp / (max_over_ranks(t64 / fs) / 1e3),
                                "ms_per_step": max_over_ranks(t64 / fs)}
        t16, _, img16, _ = time_device(ctx, torch, stream, sid, sc, "mixed_fp16", "newton", "per_pulse", fs, 1)
        forms["mixed_fp16"] = {"value": world * vp / (max_over_ranks(t16 / fs) / 1e3),
                               "ms_per_step": max_over_ranks(t16 / fs)}
        # the reference's own algorithm (grid search + mean legs, FP64) on every 20th z-slice
        gz_sub = sc.gz[::20]
        tg, _, img_grid, _ = time_device(ctx, torch, stream, sid, sc, "fp64", "grid", "mean", 1, 1, gz=gz_sub)
        img_grid = img_grid.cpu().numpy().view(np.complex128).reshape(sp.nx, sp.ny, len(gz_sub))
        nv_sub = sp.nx * sp.ny * len(gz_sub)
        forms["fp64_grid_mean_reference_algorithm"] = {
            "value": world * nv_sub * sp.n_pulses / (max_over_ranks(tg) / 1e3), "ms_per_step": max_over_ranks(tg),
            "voxels": f"{sp.nx}x{sp.ny}x{len(gz_sub)} (every 20th z-slice)"}
        forms["mixed_vs_fp64_speedup"] = value / forms["fp64_newton"]["value"]
        a = img_mixed.cpu().numpy().view(np.complex128).reshape(sp.nx, sp.ny, sp.nz)
        b = img64.cpu().numpy().view(np.complex128).reshape(sp.nx, sp.ny, sp.nz)
        c16 = img16.cpu().numpy().view(np.complex128).reshape(sp.nx, sp.ny, sp.nz)
        m = np.abs(b) >= 1e-3 * np.abs(b).max()

        def stats(x):
            return {"rel_l2": float(np.linalg.norm(x - b) / np.linalg.norm(b)),
                    "max_phase_err_rad": float(np.abs(np.angle(x[m] * np.conj(b[m]))).max()),
                    "argmax_match": bool(np.argmax(np.abs(x)) == np.argmax(np.abs(b)))}

        acc = {"mixed_vs_fp64": stats(a), "mixed_fp16_vs_fp64": stats(c16),
               "e2e_image_equals_device_image": bool(np.array_equal(img_host, a))}
        full_images = {"fp64_newton": b, "mixed": a, "mixed_fp16": c16}
        # Fermat crossing points of the mixed solver against FP64 on random (pulse, voxel) pairs
        rng = np.random.default_rng(0x5A4B0D)
        pi = rng.integers(0, sp.n_pulses, 1 << 16)
        vi = rng.integers(0, [sp.nx, sp.ny, sp.nz], size=(1 << 16, 3))
        P = np.stack([sc.gx[vi[:, 0]], sc.gy[vi[:, 1]], sc.gz[vi[:, 2]]], axis=1)
        demA = bsar.DemArrays(sc.x_vec, sc.y_vec, sc.z)
        cross = dpath = 0.0
        for ant, na, nb, first in ((sc.tx, sp.n1, sp.n2, True), (sc.rx, sp.n2, sp.n1, False)):
            p1, p2 = (ant[pi], P) if first else (P, ant[pi])
            x64 = ctx.refraction_points(demA, p1, p2, na, nb, solver="newton")
            x32 = ctx.refraction_points(demA, p1, p2, na, nb, solver="newton", precision="mixed")
            cross = max(cross, float(np.linalg.norm(x32 - x64, axis=1).max()))

            def path(X):
                return na * np.linalg.norm(p1 - X, axis=1) + nb * np.linalg.norm(p2 - X, axis=1)

            dpath = max(dpath, float(np.abs(path(x32) - path(x64)).max()))
        acc["mixed_fermat_crossing_max_err_m"] = cross
        acc["mixed_fermat_path_max_err_m"] = dpath
        acc["fermat_sample"] = "65536 random (pulse, voxel) pairs per leg, Tx->voxel and voxel->Rx"

    # ---------------- roofline of the dominant kernel (k_bp_mixed) ------------------
    peaks, peak_src = _peaks()
    l2_gbs = l2_copy_gbs(torch, stream)
    clocks = clk.summary()
    sm_mhz = peaks.get("sm_max_mhz", 1965.0)
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12          # TFLOP/s, FMA = 2 flops
    flops = fp32_flops_per_voxel_pulse(W) * vp                  # per launch
    achieved = flops / (bp_avg_ms / 1e3) / 1e12
    sfu_rate = sfu_ops_per_voxel_pulse(W) * vp / (bp_avg_ms / 1e3)
    sfu_peak = 148 * 16 * sm_mhz * 1e6
    roofline = {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                "frac": achieved / fp32_peak,
                "traffic": TRAFFIC_BYTES.get(args.config) if not args.nz else None,
                "kernel": "k_bp_mixed", "kernel_ms": bp_avg_ms,
                "peak_source": f"nominal 148 SM x 128 FP32 lanes x 2 flop x {sm_mhz:.0f} MHz (no FP32-pipe "
                               f"figure in MEASURED_PEAKS.json)",
                "sfu": {"achieved_gops": sfu_rate / 1e9, "peak_gops": sfu_peak / 1e9, "frac": sfu_rate / sfu_peak,
                        "note": "algorithmic count (both legs' rsqrt per scanned node); the warp's shared E-leg "
                                "table executes about half of them"},
                "gather": {"bytes_per_voxel_pulse": 16, "achieved_gbs": 16 * vp / (bp_avg_ms / 1e3) / 1e9,
                           "hbm_peak_gbs": peaks.get("hbm_gbs"), "peak_source": peak_src,
                           "l2_peak_gbs": l2_gbs,
                           "l2_peak_source": "measured here: device copy of a 32 MiB buffer resident in L2"},
                "fp32_flops_per_voxel_pulse": fp32_flops_per_voxel_pulse(W), "node_scan_half_width": W}

    # pulse compression (K1): HBM roofline on raw in + upsampled complex64 out
    # one compression as its own launches (inside the step it sits between back-projection
    # launches of ~0.6 s, where single-launch event times are noisy)
    pc_ms = max_over_ranks(time_compress(ctx, torch, stream, sid, "mixed"))
    ns = sp.n_samples
    pc_bytes = sp.n_pulses * (16 * ns + 8 * ns * sp.upsample)
    pc_gbs = pc_bytes / (pc_ms / 1e3) / 1e9
    roofline["pulse_compression"] = {
        "kernel": (f"k_pulse_compress_rf<{int(math.log2(ns))}>" if 4096 <= ns <= 16384 else "k_pulse_compress<float>"),
        "ms": pc_ms, "samples_per_s": sp.n_pulses * ns / (pc_ms / 1e3),
        "bytes": pc_bytes, "achieved_gbs": pc_gbs, "peak_gbs": peaks.get("hbm_gbs"), "frac": pc_gbs / peaks.get("hbm_gbs", 1),
        "flops": sp.n_pulses * 2 * (10 * ns * math.log2(ns) + 6 * ns)}
    roofline["fermat"] = {"solves_per_s": 2 * vp / (bp_avg_ms / 1e3),
                          "note": "two mixed Fermat solves per voxel-pulse inside k_bp_mixed"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        # the parity sample: the reference's own code runs on it (timed: the CPU baseline)
        # and every GPU form is compared with it or with the oracle's FP64 Newton on it
        ii, lat, hoods, groups = parity_sample(sp, sc.scat_voxel, 0x5A4B0002 + args.config)
        what = (f"{len(ii)} parity-sample voxels ({int((groups < 0).sum())} on a uniform sub-lattice "
                f"+ the 3x3x3 neighbourhoods of {len(hoods)} scatterers)")
        rate, det = cpu_reference_rate(sc, args.ref_seconds, threads, voxels=flat_voxels(sp, ii), what=what)
        cpu = {"value": rate, "unit": UNIT, "cores": det["cores"], "kind": det["kind"], "sample": det["sample"]}
        if full_images is not None:
            acc["vs_oracle_sample"] = parity_block(ctx, sid, sc, ii, lat, hoods, groups, det, full_images, W)
        del det
        shipped = min(12, threads)
        if shipped != threads:
            r12, d12 = cpu_reference_rate(sc, args.ref_seconds, shipped)
            cpu["as_shipped"] = {"value": r12, "cores": shipped,
                                 "note": "the reference caps its OpenMP loop at 12 threads"}

    config5 = None
    if rank == 0 and world == 1 and args.config == 2 and not args.no_config5 and not args.nz:
        config5 = config5_leg(ctx, torch, stream)

    serving = None
    if rank == 0 and world == 1 and args.serve_requests > 0:
        ctx.set_stream(None)
        serving = serve_leg(ctx, torch, args.serve_requests, args.serve_burst, args.serve_fp64_sample,
                            tiles=args.serve_tiles)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64 (mixed)", "data": "synthetic (seeded; no dataset)",
            "config": {"workload": workload_name(sp),
                       "form": "mixed (Newton Fermat FP32 + FP64 final step, complex64 samples, Kahan FP32 sums)",
                       "per_gpu": "one z-slab of the full grid size per rank",
                       "l2": "inputs larger than L2 (upsampled complex64 pulses "
                             f"{sp.n_pulses * sp.n_samples * sp.upsample * 8 / 2**20:.0f} MiB)",
                       "parallelism": f"voxel slabs x{world}, no collective"},
            "e2e": {"value": world * vp / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_s * 1e3, "clocks": clk_e2e.summary(),
                    "host_buffers": "pinned (raw pulses in, image out)"},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "forms": forms,
            "accuracy": acc,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "serving": serving,
            "strong_split": strong,
            "config5": config5,
        }
        print(json.dumps(line), flush=True)
    ctx.scene_release(sid)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
