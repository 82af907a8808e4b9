"""ctypes binding of libbsar.so (the C ABI declared in include/bsar.h).

This is the Python-side caller of the drop-in boundary: every method maps to one
``extern "C"`` entry point and raises :class:`BsarError` with the library's message when
the call does not return ``BSAR_OK``.  The library must exist; there is no fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent.parent          # c-_bistatic_sar_b200/
# BSAR_LIBRARY selects another build of the same library (e.g. an installed copy)
LIB_PATH = Path(os.environ.get("BSAR_LIBRARY", PKG / "lib" / "libbsar.so"))
CSRC = PKG / "csrc"

_d = C.POINTER(C.c_double)
_i64 = C.c_int64
_i32 = C.c_int32

STATUS = {0: "ok", 1: "invalid argument", 2: "HBM budget exceeded", 3: "device wait timed out",
          4: "CUDA error", 5: "not found", 6: "unsupported", 7: "queue full", 8: "cancelled"}
SOLVER = {"grid": 0, "newton": 1}
LEGS = {"mean": 0, "per_pulse": 1}
PRECISION = {"fp64": 0, "mixed": 1, "mixed_fp16": 2}
EXHAUSTIVE = 1   # BSAR_BP_EXHAUSTIVE_SCAN
FILE_LAYOUT = {"as_imager": 0, "row_major": 1}


class BsarError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Dem(C.Structure):
    _fields_ = [("nx", _i64), ("ny", _i64), ("x_vec", _d), ("y_vec", _d), ("z", _d)]


class FermatOpts(C.Structure):
    _fields_ = [("solver", _i32), ("precision", _i32), ("search_radius_m", C.c_double)]


class SceneDesc(C.Structure):
    _fields_ = [("dem", Dem), ("n_pulses", _i64), ("tx", _d), ("rx", _d), ("n_samples", _i64),
                ("samples", _d), ("samples_kind", _i32), ("upsample", _i32),
                ("n1", C.c_double), ("n2", C.c_double), ("c", C.c_double), ("fc", C.c_double),
                ("fs", C.c_double), ("chirp_f0", C.c_double), ("chirp_f1", C.c_double),
                ("chirp_T", C.c_double)]


class Grid(C.Structure):
    _fields_ = [("nx", _i64), ("ny", _i64), ("nz", _i64), ("x_axis", _d), ("y_axis", _d), ("z_axis", _d)]


class BpOpts(C.Structure):
    _fields_ = [("solver", _i32), ("legs", _i32), ("precision", _i32), ("flags", _i32),
                ("search_radius_m", C.c_double)]


class Opts(C.Structure):
    _fields_ = [("device", _i32), ("flags", _i32), ("hbm_budget_bytes", C.c_uint64)]


class MatrixHeader(C.Structure):
    _fields_ = [("ndims", C.c_uint32), ("is_complex", C.c_uint32), ("dtype_len", C.c_uint32),
                ("dtype", C.c_char * 17), ("dims", C.c_uint64 * 8), ("total", C.c_uint64)]


class ServerOpts(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("max_inflight", _i32), ("tiles_per_launch", _i32),
                ("use_graph", _i32), ("reserved", _i32), ("batch_timeout_s", C.c_double)]


class Request(C.Structure):
    _fields_ = [("scene", SceneDesc), ("scat_pos", _d), ("scat_amp", _d), ("n_scat", _i64),
                ("snr_db", C.c_double), ("seed", C.c_uint64), ("grid", Grid), ("opts", BpOpts),
                ("image_out", _d)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("launches", C.c_uint64), ("tiles", C.c_uint64), ("p50_ms", C.c_double), ("p99_ms", C.c_double),
                ("mean_ms", C.c_double), ("max_ms", C.c_double), ("voxel_pulses", C.c_double),
                ("busy_s", C.c_double), ("peak_inflight", C.c_uint64), ("peak_reserved_bytes", C.c_uint64),
                ("batch_busy_s", C.c_double)]


def build(quiet: bool = True) -> Path:
    """Compile libbsar.so for sm_100a (nvcc cross-compiles; no GPU needed)."""
    out = subprocess.run(["make", "-C", str(CSRC), "-j4"], capture_output=quiet, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"libbsar build failed:\n{out.stdout}\n{out.stderr}")
    return LIB_PATH


_LIB = None


def lib() -> C.CDLL:
    """Load libbsar.so (raises when it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise FileNotFoundError(f"{LIB_PATH} is missing: build it with bsar.native.build()")
    L = C.CDLL(str(LIB_PATH))
    V = C.c_void_p
    sigs = {
        "bsar_create": ([C.POINTER(V), C.POINTER(Opts)], _i32),
        "bsar_destroy": ([V], None),
        "bsar_status_string": ([_i32], C.c_char_p),
        "bsar_last_error": ([V], C.c_char_p),
        "bsar_set_stream": ([V, V], _i32),
        "bsar_synchronize": ([V], _i32),
        "bsar_launch_count": ([V], C.c_uint64),
        "bsar_set_tile_wait_limit": ([V, _i64], _i32),
        "bsar_bytes_in_use": ([V], C.c_uint64),
        "bsar_dem_elevation": ([V, C.POINTER(Dem), _d, _i64, _d], _i32),
        "bsar_refraction_points": ([V, C.POINTER(Dem), _d, _d, _i64, C.c_double, C.c_double,
                                    C.POINTER(FermatOpts), _d], _i32),
        "bsar_slant_range_fermat": ([V, C.POINTER(Dem), _d, _d, _i64, _d, C.c_double, C.c_double,
                                     C.POINTER(FermatOpts), _d, _d, _d, _d], _i32),
        "bsar_spline_upsample": ([V, _d, _i64, _i64, _i32, _d], _i32),
        "bsar_fft": ([V, _d, _i64, _i64, _i32], _i32),
        "bsar_fft_correlate": ([V, _d, _i64, _i64, _d, _i64, _i32, _d], _i32),
        "bsar_scene_upload": ([V, C.POINTER(SceneDesc), C.POINTER(C.c_uint64)], _i32),
        "bsar_scene_release": ([V, C.c_uint64], _i32),
        "bsar_scene_synthesize": ([V, C.POINTER(SceneDesc), _d, _d, _i64, C.c_double, C.c_uint64,
                                   C.POINTER(C.c_uint64)], _i32),
        "bsar_scene_synthesize_ex": ([V, C.POINTER(SceneDesc), _d, _d, _i64, C.c_double, C.c_uint64, _i32,
                                      C.POINTER(C.c_uint64)], _i32),
        "bsar_scene_read_samples": ([V, C.c_uint64, _d], _i32),
        "bsar_scene_compress": ([V, C.c_uint64, _i32], _i32),
        "bsar_scene_read_upsampled": ([V, C.c_uint64, _d], _i32),
        "bsar_scene_read_stored": ([V, C.c_uint64, _i32, _d], _i32),
        "bsar_backproject": ([V, C.c_uint64, C.POINTER(Grid), C.POINTER(BpOpts), _d], _i32),
        "bsar_backproject_device": ([V, C.c_uint64, C.POINTER(Grid), C.POINTER(BpOpts), V], _i32),
        "bsar_backproject_range": ([V, C.c_uint64, C.POINTER(Grid), C.POINTER(BpOpts), _i64, _i64, _d], _i32),
        "bsar_backproject_mixed_noalloc": ([V, C.c_uint64, C.POINTER(Grid), C.POINTER(BpOpts), _d], _i32),
        "bsar_matrix_read_header": ([C.c_char_p, C.POINTER(MatrixHeader)], _i32),
        "bsar_matrix_read": ([C.c_char_p, _d, C.c_uint64], _i32),
        "bsar_matrix_write": ([C.c_char_p, C.c_uint32, C.POINTER(C.c_uint64), _i32, _d], _i32),
        "bsar_scene_upload_file": ([V, C.POINTER(SceneDesc), C.c_char_p, _i32, C.POINTER(C.c_uint64)], _i32),
        "bsar_image_export": ([C.c_char_p, _d, _i64, _i64, _i64, _d, _d, _d], _i32),
        "bsar_image_export_device": ([V, C.c_char_p, V, _i64, _i64, _i64, _d, _d, _d], _i32),
        "bsar_dem_load_esri": ([C.c_char_p, C.POINTER(_i64), C.POINTER(_i64), _d, _d, _d, C.POINTER(_i32)], _i32),
        "bsar_server_create": ([V, C.POINTER(ServerOpts), C.POINTER(V)], _i32),
        "bsar_server_submit": ([V, C.POINTER(Request), C.POINTER(C.c_uint64)], _i32),
        "bsar_server_estimate": ([C.POINTER(Request), C.POINTER(C.c_uint64)], _i32),
        "bsar_server_poll": ([V, C.c_uint64, C.POINTER(_i32), _d], _i32),
        "bsar_server_wait": ([V, C.c_uint64, C.c_double, _d], _i32),
        "bsar_server_cancel": ([V, C.c_uint64], _i32),
        "bsar_server_get_stats": ([V, C.POINTER(ServerStats)], _i32),
        "bsar_server_destroy": ([V], None),
    }
    for name, (args, res) in sigs.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = L
    return L


def _f64(a, shape=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return a.reshape(shape) if shape is not None else a


def _c128(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.complex128))


def _p(a):
    return None if a is None else a.ctypes.data_as(_d)


class DemArrays:
    """Keeps the numpy arrays of a DEM alive next to its C struct."""

    def __init__(self, x_vec, y_vec, z):
        self.x = _f64(x_vec)
        self.y = _f64(y_vec)
        n = len(self.x) * len(self.y)
        self.z = _f64(z).reshape(-1)[:n] if n else np.zeros(1)
        self.c = Dem(len(self.x), len(self.y), _p(self.x), _p(self.y), _p(self.z))


class Context:
    """One bsar_ctx on a CUDA device."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self.L = lib()
        h = C.c_void_p()
        st = self.L.bsar_create(C.byref(h), C.byref(Opts(device, 0, hbm_budget_bytes)))
        if st != 0:
            raise BsarError(st, "bsar_create failed (no usable CUDA device?)")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.bsar_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _ok(self, st):
        if st != 0:
            raise BsarError(st, self.L.bsar_last_error(self.h).decode())

    # -- context ------------------------------------------------------------------------
    def set_stream(self, stream_handle: int | None):
        self._ok(self.L.bsar_set_stream(self.h, C.c_void_p(stream_handle or 0)))

    def synchronize(self):
        self._ok(self.L.bsar_synchronize(self.h))

    @property
    def launches(self) -> int:
        return int(self.L.bsar_launch_count(self.h))

    def set_tile_wait_limit(self, polls: int) -> None:
        """Polls of the mixed kernel's bounded DEM-tile wait (< 0: the default, 2^24)."""
        self._ok(self.L.bsar_set_tile_wait_limit(self.h, int(polls)))

    @property
    def bytes_in_use(self) -> int:
        return int(self.L.bsar_bytes_in_use(self.h))

    def last_error(self) -> str:
        return self.L.bsar_last_error(self.h).decode()

    # -- functional entry points -------------------------------------------------------
    def dem_elevation(self, dem: DemArrays, xy):
        xy = _f64(xy, (-1, 2))
        out = np.empty(len(xy))
        self._ok(self.L.bsar_dem_elevation(self.h, C.byref(dem.c), _p(xy), len(xy), _p(out)))
        return out

    def refraction_points(self, dem: DemArrays, p1, p2, n1, n2, solver="grid", search_radius_m=0.0,
                          precision="fp64"):
        p1 = _f64(p1, (-1, 3))
        p2 = _f64(p2, (-1, 3))
        out = np.empty((len(p1), 3))
        fo = FermatOpts(SOLVER[solver], PRECISION[precision], search_radius_m)
        self._ok(self.L.bsar_refraction_points(self.h, C.byref(dem.c), _p(p1), _p(p2), len(p1), n1, n2,
                                               C.byref(fo), _p(out)))
        return out

    def slant_range_fermat(self, dem: DemArrays, tx, rx, P, n1, n2, solver="grid", reflection=False,
                           search_radius_m=0.0):
        tx = _f64(tx, (-1, 3))
        rx = _f64(rx, (-1, 3))
        P = _f64(P, (3,))
        n = len(tx)
        ranges = np.empty((4, n))
        ida = np.empty((n, 3))
        volta = np.empty((n, 3))
        refl = np.empty((n, 3)) if reflection else None
        fo = FermatOpts(SOLVER[solver], 0, search_radius_m)
        self._ok(self.L.bsar_slant_range_fermat(self.h, C.byref(dem.c), _p(tx), _p(rx), n, _p(P), n1, n2,
                                                C.byref(fo), _p(ranges), _p(ida), _p(volta), _p(refl)))
        return ranges, ida, volta, refl

    def spline_upsample(self, data, factor=4):
        data = _c128(np.atleast_2d(data))
        b, n = data.shape
        out = np.empty((b, n * factor), dtype=np.complex128)
        self._ok(self.L.bsar_spline_upsample(self.h, _p(data.view(np.float64)), n, b, factor,
                                             _p(out.view(np.float64))))
        return out

    def fft(self, data, inverse=False):
        a = np.array(np.atleast_2d(data), dtype=np.complex128, copy=True, order="C")
        b, n = a.shape
        self._ok(self.L.bsar_fft(self.h, _p(a.view(np.float64)), n, b, 1 if inverse else 0))
        return a

    def fft_correlate(self, signal, reference, conj=True):
        s = _c128(np.atleast_2d(signal))
        r = _c128(reference)
        b, ns = s.shape
        N = max(ns, len(r))
        out = np.empty((b, N), dtype=np.complex128)
        self._ok(self.L.bsar_fft_correlate(self.h, _p(s.view(np.float64)), ns, b, _p(r.view(np.float64)),
                                           len(r), 1 if conj else 0, _p(out.view(np.float64))))
        return out

    # -- scenes ----------------------------------------------------------------------
    def scene_upload(self, dem: DemArrays, tx, rx, samples, *, kind="raw", upsample=4, n1=1.0, n2=2.0,
                     c=3e8, fc=1e9, fs=1.2e9, chirp_f0=0.0, chirp_f1=0.0, chirp_T=0.0) -> int:
        tx = _f64(tx, (-1, 3))
        rx = _f64(rx, (-1, 3))
        smp = _c128(samples)
        desc = SceneDesc(dem.c, len(tx), _p(tx), _p(rx), smp.shape[1], _p(smp.view(np.float64)),
                         0 if kind == "raw" else 1, upsample, n1, n2, c, fc, fs, chirp_f0, chirp_f1, chirp_T)
        sid = C.c_uint64()
        self._ok(self.L.bsar_scene_upload(self.h, C.byref(desc), C.byref(sid)))
        return int(sid.value)

    def scene_synthesize(self, dem: DemArrays, tx, rx, n_samples, scat_pos, scat_amp, *, snr_db=float("inf"),
                         seed=0, upsample=4, n1=1.0, n2=2.0, c=3e8, fc=1e9, fs=1.2e9, chirp_f0=0.0, chirp_f1=0.0,
                         chirp_T=0.0, reference_bins=False) -> int:
        """Resident raw scene with echoes synthesised on the device (bsar_scene_synthesize);
        reference_bins: the simulator's integer echo bin and circular wrap."""
        tx = _f64(tx, (-1, 3))
        rx = _f64(rx, (-1, 3))
        pos = _f64(scat_pos, (-1, 3))
        amp = _f64(scat_amp)
        desc = SceneDesc(dem.c, len(tx), _p(tx), _p(rx), int(n_samples), None, 0, upsample, n1, n2, c, fc, fs,
                         chirp_f0, chirp_f1, chirp_T)
        sid = C.c_uint64()
        self._ok(self.L.bsar_scene_synthesize_ex(self.h, C.byref(desc), _p(pos), _p(amp), len(amp), snr_db,
                                                 seed & (2**64 - 1), 1 if reference_bins else 0, C.byref(sid)))
        return int(sid.value)

    def scene_upload_file(self, dem: DemArrays, tx, rx, path, *, layout="as_imager", kind="compressed", upsample=4,
                          n1=1.0, n2=2.0, c=3e8, fc=1e9, fs=1.2e9, chirp_f0=0.0, chirp_f1=0.0, chirp_T=0.0) -> int:
        """Resident scene whose pulses come from a matrix file (bsar_scene_upload_file):
        layout "as_imager" (the imager's reading) or "row_major" (transposed on the GPU)."""
        tx = _f64(tx, (-1, 3))
        rx = _f64(rx, (-1, 3))
        desc = SceneDesc(dem.c, len(tx), _p(tx), _p(rx), 0, None, 0 if kind == "raw" else 1, upsample, n1, n2, c, fc,
                         fs, chirp_f0, chirp_f1, chirp_T)
        sid = C.c_uint64()
        self._ok(self.L.bsar_scene_upload_file(self.h, C.byref(desc), str(path).encode(), FILE_LAYOUT[layout],
                                               C.byref(sid)))
        return int(sid.value)

    def image_export_device(self, path, d_image_ptr: int, nx: int, ny: int, nz: int, gx=None, gy=None, gz=None):
        """Write a device image ([x][y][z] complex128) in the reference's file order."""
        ax = [None if a is None else _f64(a) for a in (gx, gy, gz)]
        self._ok(self.L.bsar_image_export_device(self.h, str(path).encode(), C.c_void_p(d_image_ptr), nx, ny, nz,
                                                 *[_p(a) for a in ax]))

    def scene_read_samples(self, sid: int, n_pulses: int, n_samples: int):
        out = np.empty((n_pulses, n_samples), dtype=np.complex128)
        self._ok(self.L.bsar_scene_read_samples(self.h, sid, _p(out.view(np.float64))))
        return out

    def scene_release(self, sid: int):
        self._ok(self.L.bsar_scene_release(self.h, sid))

    def scene_compress(self, sid: int, precision="fp64"):
        self._ok(self.L.bsar_scene_compress(self.h, sid, PRECISION[precision]))

    def scene_read_upsampled(self, sid: int, n_pulses: int, n_out: int):
        out = np.empty((n_pulses, n_out), dtype=np.complex128)
        self._ok(self.L.bsar_scene_read_upsampled(self.h, sid, _p(out.view(np.float64))))
        return out

    def scene_read_stored(self, sid: int, n_pulses: int, n_out: int, precision="fp64"):
        """Upsampled pulses as stored for `precision`, widened to complex128."""
        out = np.empty((n_pulses, n_out), dtype=np.complex128)
        self._ok(self.L.bsar_scene_read_stored(self.h, sid, PRECISION[precision], _p(out.view(np.float64))))
        return out

    @staticmethod
    def _grid(gx, gy, gz):
        gx, gy, gz = _f64(gx), _f64(gy), _f64(gz)
        return (gx, gy, gz), Grid(len(gx), len(gy), len(gz), _p(gx), _p(gy), _p(gz))

    def backproject(self, sid: int, gx, gy, gz, *, solver="grid", legs="mean", precision="fp64",
                    search_radius_m=0.0, out=None, exhaustive=False):
        """Image [x][y][z] complex128; `out` (C-contiguous complex128 of that shape, e.g.
        a view of pinned memory) receives it instead of a new array.  `exhaustive`: the
        mixed forms rank every node of each node-scan window (BSAR_BP_EXHAUSTIVE_SCAN;
        the same image, slower)."""
        keep, g = self._grid(gx, gy, gz)
        o = BpOpts(SOLVER[solver], LEGS[legs], PRECISION[precision], EXHAUSTIVE if exhaustive else 0,
                   search_radius_m)
        if out is None:
            out = np.empty((g.nx, g.ny, g.nz), dtype=np.complex128)
        elif out.shape != (g.nx, g.ny, g.nz) or out.dtype != np.complex128 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous complex128 array of the grid's shape")
        self._ok(self.L.bsar_backproject(self.h, sid, C.byref(g), C.byref(o), _p(out.view(np.float64))))
        return out

    def backproject_range(self, sid: int, gx, gy, gz, v_begin: int, v_count: int, *, solver="grid", legs="mean",
                          precision="fp64", search_radius_m=0.0, exhaustive=False):
        """Voxels [v_begin, v_begin + v_count) of the grid's flat order (z -> x -> y) in the
        full (nx, ny, nz) image, the others 0; each value equals backproject's."""
        keep, g = self._grid(gx, gy, gz)
        o = BpOpts(SOLVER[solver], LEGS[legs], PRECISION[precision], EXHAUSTIVE if exhaustive else 0,
                   search_radius_m)
        out = np.empty((g.nx, g.ny, g.nz), dtype=np.complex128)
        self._ok(self.L.bsar_backproject_range(self.h, sid, C.byref(g), C.byref(o), int(v_begin), int(v_count),
                                               _p(out.view(np.float64))))
        return out

    def backproject_mixed_noalloc(self, sid: int, gx, gy, gz, *, precision="mixed", search_radius_m=0.0,
                                  exhaustive=False):
        """Mixed back-projection that allocates no GPU memory, for callers whose GPU memory
        belongs to another allocator: a fixed 64 MiB per-device scratch, one call at a
        time per device; the scene must already be compressed for `precision`."""
        keep, g = self._grid(gx, gy, gz)
        o = BpOpts(SOLVER["newton"], LEGS["per_pulse"], PRECISION[precision], EXHAUSTIVE if exhaustive else 0,
                   search_radius_m)
        out = np.empty((g.nx, g.ny, g.nz), dtype=np.complex128)
        self._ok(self.L.bsar_backproject_mixed_noalloc(self.h, sid, C.byref(g), C.byref(o), _p(out.view(np.float64))))
        return out

    def backproject_device(self, sid: int, gx, gy, gz, d_image_ptr: int, *, solver="grid", legs="mean",
                           precision="fp64", search_radius_m=0.0, exhaustive=False):
        keep, g = self._grid(gx, gy, gz)
        o = BpOpts(SOLVER[solver], LEGS[legs], PRECISION[precision], EXHAUSTIVE if exhaustive else 0,
                   search_radius_m)
        self._ok(self.L.bsar_backproject_device(self.h, sid, C.byref(g), C.byref(o), C.c_void_p(d_image_ptr)))


def synthesize_scene(ctx: Context, scene, snr_db=None, seed=None) -> int:
    """Resident raw scene for a bsar.scene.Scene whose echoes are synthesised on the GPU
    (the scene's DEM, trajectories and scatterers; its numpy `raw` is not used)."""
    sp = scene.spec
    dem = DemArrays(scene.x_vec, scene.y_vec, scene.z)
    f0, f1 = -sp.bandwidth / 2.0, sp.bandwidth / 2.0
    return ctx.scene_synthesize(dem, scene.tx, scene.rx, sp.n_samples, scene.scat_pos, scene.scat_amp,
                                snr_db=sp.snr_db if snr_db is None else snr_db,
                                seed=sp.seed if seed is None else seed, upsample=sp.upsample, n1=sp.n1, n2=sp.n2,
                                c=3e8, fc=sp.fc, fs=sp.fs, chirp_f0=f0, chirp_f1=f1, chirp_T=sp.pulse_T)


def upload_scene(ctx: Context, scene, kind="raw") -> int:
    """Upload a bsar.scene.Scene (raw echoes) to the context."""
    sp = scene.spec
    dem = DemArrays(scene.x_vec, scene.y_vec, scene.z)
    f0, f1 = -sp.bandwidth / 2.0, sp.bandwidth / 2.0
    return ctx.scene_upload(dem, scene.tx, scene.rx, scene.raw, kind=kind, upsample=sp.upsample,
                            n1=sp.n1, n2=sp.n2, c=3e8, fc=sp.fc, fs=sp.fs, chirp_f0=f0, chirp_f1=f1,
                            chirp_T=sp.pulse_T)


def _request(dem: DemArrays, tx, rx, gx, gy, gz, *, samples=None, n_samples=None, kind="raw", scat_pos=None,
             scat_amp=None, snr_db=float("inf"), seed=0, upsample=4, n1=1.0, n2=2.0, c=3e8, fc=1e9, fs=1.2e9,
             chirp_f0=0.0, chirp_f1=0.0, chirp_T=0.0, precision="mixed", search_radius_m=0.0, exhaustive=False):
    """bsar_request for the server, the output image and the arrays the request points into."""
    tx = _f64(tx, (-1, 3))
    rx = _f64(rx, (-1, 3))
    keep = [dem, tx, rx]
    if samples is not None:
        smp = _c128(samples)
        keep.append(smp)
        ns, sp = smp.shape[1], _p(smp.view(np.float64))
        pos = amp = None
        nscat = 0
    else:
        ns, sp = int(n_samples), None
        pos = _f64(scat_pos, (-1, 3))
        amp = _f64(scat_amp)
        keep += [pos, amp]
        nscat = len(amp)
    desc = SceneDesc(dem.c, len(tx), _p(tx), _p(rx), ns, sp, 0 if kind == "raw" else 1, upsample, n1, n2, c, fc, fs,
                     chirp_f0, chirp_f1, chirp_T)
    axes, g = Context._grid(gx, gy, gz)
    keep.append(axes)
    out = np.empty((g.nx, g.ny, g.nz), dtype=np.complex128)
    o = BpOpts(SOLVER["newton"], LEGS["per_pulse"], PRECISION[precision], EXHAUSTIVE if exhaustive else 0,
               search_radius_m)
    req = Request(desc, _p(pos), _p(amp), nscat, snr_db, seed & (2**64 - 1), g, o, _p(out.view(np.float64)))
    return req, out, keep


class Server:
    """Continuous-batching image-formation server on a context (bsar_server_*).

    ``submit`` copies the small arrays; the raw samples (if any) and the output image
    are kept alive here until the request completes."""

    def __init__(self, ctx: Context, *, hbm_budget_bytes=0, max_inflight=64, tiles_per_launch=0, use_graph=True,
                 batch_timeout_s=0.0):
        self.ctx = ctx
        self.L = ctx.L
        h = C.c_void_p()
        st = self.L.bsar_server_create(ctx.h, C.byref(ServerOpts(hbm_budget_bytes, max_inflight, tiles_per_launch,
                                                                  1 if use_graph else 0, 0, batch_timeout_s)),
                                       C.byref(h))
        if st != 0:
            raise BsarError(st, ctx.last_error())
        self.h = h
        self._live = {}

    def close(self):
        if getattr(self, "h", None):
            self.L.bsar_server_destroy(self.h)
            self.h = None
            self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, dem: DemArrays, tx, rx, gx, gy, gz, **kw) -> int:
        """Queue one image; echoes come from `samples` or are synthesised on the device
        from `scat_pos`/`scat_amp` (then `n_samples` gives the pulse length).  Keyword
        arguments as in :func:`_request`."""
        req, out, keep = _request(dem, tx, rx, gx, gy, gz, **kw)
        rid = C.c_uint64()
        st = self.L.bsar_server_submit(self.h, C.byref(req), C.byref(rid))
        if st != 0:
            raise BsarError(st, "request rejected")
        self._live[int(rid.value)] = (out, keep)
        return int(rid.value)

    @staticmethod
    def estimate(dem: DemArrays, tx, rx, gx, gy, gz, **kw) -> int:
        """Device bytes the request would reserve against a server's budget."""
        req, _, _ = _request(dem, tx, rx, gx, gy, gz, **kw)
        b = C.c_uint64()
        st = lib().bsar_server_estimate(C.byref(req), C.byref(b))
        if st != 0:
            raise BsarError(st, "estimate")
        return int(b.value)

    def poll(self, rid: int):
        """(done, latency_ms); raises when the request failed."""
        done = _i32()
        lat = C.c_double()
        st = self.L.bsar_server_poll(self.h, rid, C.byref(done), C.byref(lat))
        if st != 0:
            raise BsarError(st, f"request {rid} failed")
        return bool(done.value), float(lat.value)

    def wait(self, rid: int, timeout_s: float = 600.0):
        """Image and latency (ms) of a request; raises when it failed or timed out."""
        lat = C.c_double()
        st = self.L.bsar_server_wait(self.h, rid, timeout_s, C.byref(lat))
        if st != 0:
            raise BsarError(st, f"request {rid}")
        out, _ = self._live.pop(rid)
        return out, float(lat.value)

    def cancel(self, rid: int) -> None:
        """bsar_server_cancel: the request completes with BSAR_ERR_CANCELLED."""
        st = self.L.bsar_server_cancel(self.h, rid)
        if st != 0:
            raise BsarError(st, f"cancel {rid}")

    def stats(self) -> dict:
        o = ServerStats()
        st = self.L.bsar_server_get_stats(self.h, C.byref(o))
        if st != 0:
            raise BsarError(st, "stats")
        return {k: getattr(o, k) for k, _ in ServerStats._fields_}


def submit_scene(server: Server, scene, gx, gy, gz, *, synthesize=True, precision="mixed", snr_db=None, seed=None):
    """Queue a bsar.scene.Scene on a server: echoes synthesised on the device from the
    scene's scatterers (default) or uploaded from its numpy `raw`."""
    sp = scene.spec
    dem = DemArrays(scene.x_vec, scene.y_vec, scene.z)
    f0, f1 = -sp.bandwidth / 2.0, sp.bandwidth / 2.0
    common = dict(upsample=sp.upsample, n1=sp.n1, n2=sp.n2, c=3e8, fc=sp.fc, fs=sp.fs, chirp_f0=f0, chirp_f1=f1,
                  chirp_T=sp.pulse_T, precision=precision)
    if synthesize:
        return server.submit(dem, scene.tx, scene.rx, gx, gy, gz, n_samples=sp.n_samples, scat_pos=scene.scat_pos,
                             scat_amp=scene.scat_amp, snr_db=sp.snr_db if snr_db is None else snr_db,
                             seed=sp.seed if seed is None else seed, **common)
    return server.submit(dem, scene.tx, scene.rx, gx, gy, gz, samples=scene.raw, **common)


# ---- files (no context needed) --------------------------------------------------------
def matrix_read(path):
    """readBinary of a matrix file: (complex128 values, dims, is_complex)."""
    L = lib()
    h = MatrixHeader()
    st = L.bsar_matrix_read_header(str(path).encode(), C.byref(h))
    if st != 0:
        raise BsarError(st, f"cannot read the header of {path}")
    out = np.empty(max(int(h.total), 1), dtype=np.complex128)
    st = L.bsar_matrix_read(str(path).encode(), _p(out.view(np.float64)), int(h.total))
    if st != 0:
        raise BsarError(st, f"cannot read {path}")
    return out[: int(h.total)], [int(h.dims[k]) for k in range(h.ndims)], bool(h.is_complex)


def matrix_write(path, data):
    """exportComplexMatrix-style file of a complex (or real) array of any rank."""
    a = np.asarray(data)
    cplx = np.iscomplexobj(a)
    a = np.ascontiguousarray(a, dtype=np.complex128 if cplx else np.float64)
    dims = (C.c_uint64 * max(a.ndim, 1))(*a.shape)
    st = lib().bsar_matrix_write(str(path).encode(), a.ndim, dims, 1 if cplx else 0, _p(a.view(np.float64)))
    if st != 0:
        raise BsarError(st, f"cannot write {path}")


def image_export(path, image, gx=None, gy=None, gz=None):
    """export3DComplexMatrix of an [x][y][z] complex image (x fastest in the file)."""
    img = _c128(image)
    nx, ny, nz = img.shape
    ax = [None if a is None else _f64(a) for a in (gx, gy, gz)]
    st = lib().bsar_image_export(str(path).encode(), _p(img.view(np.float64)), nx, ny, nz, *[_p(a) for a in ax])
    if st != 0:
        raise BsarError(st, f"cannot write {path}")


def dem_load_esri(path):
    """loadDEM of an ESRI ASCII grid: (x_vec, y_vec, z[ny, nx], flags)."""
    L = lib()
    nx, ny, fl = _i64(), _i64(), _i32()
    st = L.bsar_dem_load_esri(str(path).encode(), C.byref(nx), C.byref(ny), None, None, None, C.byref(fl))
    if st != 0:
        raise BsarError(st, f"cannot load {path}")
    x = np.empty(max(nx.value, 1))
    y = np.empty(max(ny.value, 1))
    z = np.empty(max(nx.value * ny.value, 1))
    st = L.bsar_dem_load_esri(str(path).encode(), C.byref(nx), C.byref(ny), _p(x), _p(y), _p(z), C.byref(fl))
    if st != 0:
        raise BsarError(st, f"cannot load {path}")
    return x[: nx.value], y[: ny.value], z[: nx.value * ny.value].reshape(ny.value, nx.value), int(fl.value)
