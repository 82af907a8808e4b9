"""ctypes front end of the parity oracle -- TEST INFRASTRUCTURE ONLY.

Two CPU libraries sit behind this module:

* ``libbsar_oracle.so`` -- ``bsar_oracle.c``, the C restatement of the reference's hot
  path (grid-search Fermat, bilinear DEM, Hermite upsampling, radix-2 FFT, inline
  back-projection) plus the FP64 Newton solver the product's Newton kernels follow.
* ``_ref/libbsar_ref.so`` -- the reference's own ``src/*.cpp`` compiled unmodified,
  with ``ref_harness.cpp`` (built only where the reference tree is present).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline / reference legs of
``bench.py`` import this module.  Arrays are numpy; complex arrays are complex128.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "libbsar_oracle.so"
REF_SO = HERE / "_ref" / "libbsar_ref.so"
# the reference checkout: $BSAR_REFERENCE_TREE, else a `reference` directory beside the
# repository
REF_TREE = Path(os.environ.get("BSAR_REFERENCE_TREE", str(HERE.parent.parent / "reference")))

_d = C.POINTER(C.c_double)
_i64 = C.c_int64
_i32 = C.c_int32


def build(ref: bool = True) -> None:
    """Compile the restatement (always) and the reference objects (when the tree exists)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    if ref and (REF_TREE / "src" / "raw_data_processing.cpp").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={REF_TREE}"], check=True)


def _ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(_d)


def _f64(a, shape=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    if shape is not None:
        a = a.reshape(shape)
    return a


def _c2r(a):
    """complex128 array -> contiguous interleaved float64 view."""
    a = np.ascontiguousarray(np.asarray(a, dtype=np.complex128))
    return a.view(np.float64)


class _BoDem(C.Structure):
    _fields_ = [("nx", _i64), ("ny", _i64), ("xv", _d), ("yv", _d), ("z", _d),
                ("empty", _i32), ("pad", _i32)]


class _BoBpArgs(C.Structure):
    _fields_ = [("dem", C.POINTER(_BoDem)), ("tx", _d), ("rx", _d), ("np", _i64),
                ("rc", _d), ("nr", _i64), ("gx", _d), ("gy", _d), ("gz", _d),
                ("nx", _i64), ("ny", _i64), ("nz", _i64),
                ("n1", C.c_double), ("n2", C.c_double), ("c", C.c_double),
                ("fs_eff", C.c_double), ("lam", C.c_double),
                ("legs", _i32), ("solver", _i32), ("search_nodes", _i32), ("pad", _i32)]


class Dem:
    """DEM in the oracle's packed layout: z[j, i] = Z_DEM[j][i] (rows follow y_vec)."""

    def __init__(self, x_vec, y_vec, z):
        self.x = _f64(x_vec)
        self.y = _f64(y_vec)
        self.z = _f64(z, (len(self.y), len(self.x))) if len(self.x) and len(self.y) else np.zeros((0,))
        self.c = _BoDem(len(self.x), len(self.y), _ptr(self.x), _ptr(self.y), _ptr(self.z),
                        1 if (len(self.x) == 0 or len(self.y) == 0) else 0, 0)


class Oracle:
    """The C restatement (always available once built)."""

    def __init__(self, path: Path = ORACLE_SO):
        if not Path(path).exists():
            build(ref=False)
        L = C.CDLL(str(path))
        self.L = L
        L.bo_dem_elevation_batch.argtypes = [C.POINTER(_BoDem), _d, _i64, _d]
        L.bo_refraction_grid.argtypes = [C.c_double] * 6 + [C.POINTER(_BoDem), C.c_double, C.c_double, _d]
        L.bo_refraction_newton.argtypes = [C.c_double] * 6 + [C.POINTER(_BoDem), C.c_double,
                                                               C.c_double, _i32, _d]
        L.bo_slant_range_fermat.argtypes = [C.POINTER(_BoDem), _d, _d, _i64, _d, C.c_double,
                                            C.c_double, _i32, _i32, _d, _d, _d, _d]
        L.bo_spline_upsample_batch.argtypes = [_d, _i64, _i64, _i32, _d]
        L.bo_fft.argtypes = [_d, _i64]
        L.bo_ifft.argtypes = [_d, _i64]
        L.bo_fft_correlate_batch.argtypes = [_d, _i64, _i64, _d, _i64, _i32, _d]
        L.bo_create_chirp.argtypes = [C.c_double] * 4 + [_d, _i64]
        L.bo_create_chirp.restype = _i64
        L.bo_matched_reference.argtypes = [_d, _i64, _i64, _d]
        L.bo_backproject.argtypes = [C.POINTER(_BoBpArgs), C.POINTER(_i64), _i64, _d]

    # -- DEM / Fermat ---------------------------------------------------------------
    def dem_elevation(self, dem: Dem, xy):
        xy = _f64(xy, (-1, 2))
        out = np.empty(len(xy))
        self.L.bo_dem_elevation_batch(C.byref(dem.c), _ptr(xy), len(xy), _ptr(out))
        return out

    def refraction_points(self, dem: Dem, p1, p2, n1, n2, solver="grid", search_nodes=6):
        p1 = _f64(p1, (-1, 3))
        p2 = _f64(p2, (-1, 3))
        out = np.empty((len(p1), 3))
        o = np.empty(3)
        for k in range(len(p1)):
            if solver == "grid":
                self.L.bo_refraction_grid(*p1[k], *p2[k], C.byref(dem.c), n1, n2, _ptr(o))
            else:
                self.L.bo_refraction_newton(*p1[k], *p2[k], C.byref(dem.c), n1, n2, search_nodes,
                                            _ptr(o))
            out[k] = o
        return out

    def slant_range_fermat(self, dem: Dem, tx, rx, P, n1, n2, solver="grid", reflection=False,
                           search_nodes=6):
        tx = _f64(tx, (-1, 3))
        rx = _f64(rx, (-1, 3))
        P = _f64(P, (3,))
        n = len(tx)
        ranges = np.empty((4, n))
        ida = np.empty((n, 3))
        volta = np.empty((n, 3))
        refl = np.empty((n, 3)) if reflection else None
        self.L.bo_slant_range_fermat(C.byref(dem.c), _ptr(tx), _ptr(rx), n, _ptr(P), n1, n2,
                                     0 if solver == "grid" else 1, search_nodes, _ptr(ranges), _ptr(ida),
                                     _ptr(volta), _ptr(refl))
        return ranges, ida, volta, refl

    # -- signal -----------------------------------------------------------------------
    def spline_upsample(self, data, factor=4):
        data = np.ascontiguousarray(np.atleast_2d(np.asarray(data, dtype=np.complex128)))
        b, n = data.shape
        out = np.empty((b, n * factor), dtype=np.complex128)
        self.L.bo_spline_upsample_batch(_ptr(_c2r(data)), n, b, factor, _ptr(out.view(np.float64)))
        return out

    def fft(self, data, inverse=False):
        a = np.array(data, dtype=np.complex128, copy=True)
        (self.L.bo_ifft if inverse else self.L.bo_fft)(_ptr(a.view(np.float64)), len(a))
        return a

    def fft_correlate(self, signal, reference, conj=True):
        s = np.ascontiguousarray(np.atleast_2d(np.asarray(signal, dtype=np.complex128)))
        r = np.ascontiguousarray(np.asarray(reference, dtype=np.complex128))
        b, ns = s.shape
        N = max(ns, len(r))
        out = np.empty((b, N), dtype=np.complex128)
        self.L.bo_fft_correlate_batch(_ptr(s.view(np.float64)), ns, b, _ptr(r.view(np.float64)),
                                      len(r), 1 if conj else 0, _ptr(out.view(np.float64)))
        return out

    def create_chirp(self, f0, f1, T, fs):
        n = int(T * fs) + 1
        out = np.empty(n, dtype=np.complex128)
        self.L.bo_create_chirp(f0, f1, T, fs, _ptr(out.view(np.float64)), n)
        return out

    def matched_reference(self, chirp, nmax):
        chirp = np.ascontiguousarray(chirp, dtype=np.complex128)
        out = np.empty(nmax, dtype=np.complex128)
        self.L.bo_matched_reference(_ptr(chirp.view(np.float64)), len(chirp), nmax,
                                    _ptr(out.view(np.float64)))
        return out

    # -- back-projection ------------------------------------------------------------
    def backproject(self, dem: Dem, tx, rx, rc, gx, gy, gz, n1, n2, c, fs_eff, lam,
                    legs="mean", solver="grid", voxels=None, search_nodes=6):
        tx = _f64(tx, (-1, 3))
        rx = _f64(rx, (-1, 3))
        rc = np.ascontiguousarray(np.asarray(rc, dtype=np.complex128))
        gx, gy, gz = _f64(gx), _f64(gy), _f64(gz)
        args = _BoBpArgs(C.pointer(dem.c), _ptr(tx), _ptr(rx), len(tx), _ptr(rc.view(np.float64)),
                         rc.shape[1], _ptr(gx), _ptr(gy), _ptr(gz), len(gx), len(gy), len(gz),
                         n1, n2, c, fs_eff, lam, 0 if legs == "mean" else 1,
                         0 if solver == "grid" else 1, search_nodes, 0)
        if voxels is None:
            out = np.empty((len(gx), len(gy), len(gz)), dtype=np.complex128)
            self.L.bo_backproject(C.byref(args), None, 0, _ptr(out.view(np.float64)))
        else:
            v = np.ascontiguousarray(voxels, dtype=np.int64)
            out = np.empty(len(v), dtype=np.complex128)
            self.L.bo_backproject(C.byref(args), v.ctypes.data_as(C.POINTER(_i64)), len(v),
                                  _ptr(out.view(np.float64)))
        return out


class Reference:
    """The reference's own compiled functions (oracle/_ref/libbsar_ref.so)."""

    @staticmethod
    def available() -> bool:
        return REF_SO.exists()

    def __init__(self, path: Path = REF_SO):
        L = C.CDLL(str(path))
        self.L = L
        dem5 = [_i64, _i64, _d, _d, _d]
        L.ref_dem_elevation.argtypes = dem5 + [_d, _i64, _d]
        L.ref_refraction_points.argtypes = dem5 + [_d, _d, _i64, C.c_double, C.c_double, _d]
        L.ref_slant_range_fermat.argtypes = dem5 + [_d, _d, _i64, _d, C.c_double, C.c_double,
                                                    _d, _d, _d, _d]
        L.ref_spline_upsample.argtypes = [_d, _i64, _i64, _i32, _d]
        L.ref_fft.argtypes = [_d, _i64, _i32]
        L.ref_fft_correlate_batch.argtypes = [_d, _i64, _i64, _d, _i64, _i32, _i32, _d]
        L.ref_create_chirp.argtypes = [C.c_double] * 4 + [_d, _i64]
        L.ref_create_chirp.restype = _i64
        L.ref_read_binary.argtypes = [C.c_char_p, C.POINTER(C.c_uint64), C.POINTER(_i32), C.POINTER(_i32), _d, _i64]
        L.ref_read_binary.restype = _i64
        L.ref_export_complex_matrix.argtypes = [C.c_char_p, _i64, _i64, _d]
        L.ref_export_3d.argtypes = [C.c_char_p, _i64, _i64, _i64, _d, _d, _d, _d]
        L.ref_load_dem.argtypes = [C.c_char_p, C.POINTER(_i64), C.POINTER(_i64), _d, _d, _d]
        L.ref_process_raw_data.argtypes = ([_i64, _d, _d, _d, _d] + [C.c_double] * 7 +
                                           [_i32, C.c_double, C.c_double, _d, _d, _d, _d, _i64])
        L.ref_process_raw_data.restype = _i64
        L.ref_backproject.argtypes = dem5 + [_d, _d, _i64, _d, _i64, _d, _i64, _d, _i64, _d, _i64,
                                             C.c_double, C.c_double, C.c_double, C.c_double,
                                             C.c_double, _i32, C.POINTER(_i64), _i64, _i32, _d]

    @staticmethod
    def _dem(dem: Dem):
        return [len(dem.x), len(dem.y), _ptr(dem.x), _ptr(dem.y), _ptr(dem.z)]

    def dem_elevation(self, dem: Dem, xy):
        xy = _f64(xy, (-1, 2))
        out = np.empty(len(xy))
        self.L.ref_dem_elevation(*self._dem(dem), _ptr(xy), len(xy), _ptr(out))
        return out

    def refraction_points(self, dem: Dem, p1, p2, n1, n2):
        p1 = _f64(p1, (-1, 3))
        p2 = _f64(p2, (-1, 3))
        out = np.empty((len(p1), 3))
        self.L.ref_refraction_points(*self._dem(dem), _ptr(p1), _ptr(p2), len(p1), n1, n2, _ptr(out))
        return out

    def slant_range_fermat(self, dem: Dem, tx, rx, P, n1, n2):
        tx = _f64(tx, (-1, 3))
        rx = _f64(rx, (-1, 3))
        P = _f64(P, (3,))
        n = len(tx)
        ranges = np.empty((4, n))
        ida = np.empty((n, 3))
        volta = np.empty((n, 3))
        refl = np.empty((n, 3))
        self.L.ref_slant_range_fermat(*self._dem(dem), _ptr(tx), _ptr(rx), n, _ptr(P), n1, n2,
                                      _ptr(ranges), _ptr(ida), _ptr(volta), _ptr(refl))
        return ranges, ida, volta, refl

    def spline_upsample(self, data, factor=4):
        data = np.ascontiguousarray(np.atleast_2d(np.asarray(data, dtype=np.complex128)))
        b, n = data.shape
        out = np.empty((b, n * factor), dtype=np.complex128)
        self.L.ref_spline_upsample(_ptr(data.view(np.float64)), n, b, factor, _ptr(out.view(np.float64)))
        return out

    def fft(self, data, inverse=False):
        a = np.array(data, dtype=np.complex128, copy=True)
        self.L.ref_fft(_ptr(a.view(np.float64)), len(a), 1 if inverse else 0)
        return a

    def fft_correlate(self, signal, reference, conj=True, nthreads=0):
        s = np.ascontiguousarray(np.atleast_2d(np.asarray(signal, dtype=np.complex128)))
        r = np.ascontiguousarray(np.asarray(reference, dtype=np.complex128))
        b, ns = s.shape
        N = max(ns, len(r))
        out = np.empty((b, N), dtype=np.complex128)
        self.L.ref_fft_correlate_batch(_ptr(s.view(np.float64)), ns, b, _ptr(r.view(np.float64)),
                                       len(r), 1 if conj else 0, nthreads, _ptr(out.view(np.float64)))
        return out

    def create_chirp(self, f0, f1, T, fs):
        n = int(T * fs) + 1
        out = np.empty(n, dtype=np.complex128)
        got = self.L.ref_create_chirp(f0, f1, T, fs, _ptr(out.view(np.float64)), n)
        return out[:got]

    def process_raw_data(self, tx, rx, P, ranges, f0, f1, T, fs, lamb, rcs, c, M, n1, n2):
        """processRawData on given ranges (4 x np: r1Tx, r2Tx, r1Rx, r2Rx); returns the
        pulse-major (np x M) aux, raw and root matrices and the chirp."""
        tx = _f64(tx, (-1, 3))
        rx = _f64(rx, (-1, 3))
        P = _f64(P, (3,))
        ranges = _f64(ranges, (4, -1))
        n = len(tx)
        aux, raw, root = (np.empty((n, M), dtype=np.complex128) for _ in range(3))
        cap = int(T * fs) + 2
        chirp = np.empty(cap, dtype=np.complex128)
        got = self.L.ref_process_raw_data(n, _ptr(tx), _ptr(rx), _ptr(P), _ptr(ranges), f0, f1, T, fs, lamb, rcs, c,
                                          M, n1, n2, _ptr(aux.view(np.float64)), _ptr(raw.view(np.float64)),
                                          _ptr(root.view(np.float64)), _ptr(chirp.view(np.float64)), cap)
        return aux, raw, root, chirp[:got]

    def backproject(self, dem: Dem, tx, rx, rc, gx, gy, gz, n1, n2, c, fs_eff, lam,
                    legs="mean", voxels=None, nthreads=0):
        tx = _f64(tx, (-1, 3))
        rx = _f64(rx, (-1, 3))
        rc = np.ascontiguousarray(np.asarray(rc, dtype=np.complex128))
        gx, gy, gz = _f64(gx), _f64(gy), _f64(gz)
        np_ = len(tx)
        if voxels is None:
            out = np.empty((len(gx), len(gy), len(gz)), dtype=np.complex128)
            vp, nv = None, 0
        else:
            v = np.ascontiguousarray(voxels, dtype=np.int64)
            out = np.empty(len(v), dtype=np.complex128)
            vp, nv = v.ctypes.data_as(C.POINTER(_i64)), len(v)
        self.L.ref_backproject(*self._dem(dem), _ptr(tx), _ptr(rx), np_, _ptr(rc.view(np.float64)),
                               rc.shape[1], _ptr(gx), len(gx), _ptr(gy), len(gy), _ptr(gz), len(gz),
                               n1, n2, c, fs_eff, lam, 0 if legs == "mean" else 1, vp, nv,
                               nthreads, _ptr(out.view(np.float64)))
        return out


def _ref_files_methods():
    """File readers / writers of the reference (binary_reader.cpp, data_export.cpp,
    load_dem_simple.cpp) on the Reference class."""

    def read_binary(self, path, cap=1 << 26):
        dims = (C.c_uint64 * 8)()
        nd, cx = _i32(), _i32()
        out = np.empty(cap, dtype=np.complex128)
        n = self.L.ref_read_binary(str(path).encode(), dims, C.byref(nd), C.byref(cx), _ptr(out.view(np.float64)), cap)
        if n < 0:
            raise RuntimeError(f"reference readBinary failed on {path}")
        return out[:n].copy(), [int(dims[k]) for k in range(nd.value)], bool(cx.value)

    def export_complex_matrix(self, path, m):
        m = np.ascontiguousarray(np.asarray(m, dtype=np.complex128))
        self.L.ref_export_complex_matrix(str(path).encode(), m.shape[0], m.shape[1], _ptr(m.view(np.float64)))

    def export_3d(self, path, img, gx=None, gy=None, gz=None):
        img = np.ascontiguousarray(np.asarray(img, dtype=np.complex128))
        nx, ny, nz = img.shape
        ax = [None if a is None else _f64(a) for a in (gx, gy, gz)]
        self.L.ref_export_3d(str(path).encode(), nx, ny, nz, _ptr(img.view(np.float64)),
                             *[None if a is None else _ptr(a) for a in ax])

    def load_dem(self, path):
        nx, ny = _i64(), _i64()
        self.L.ref_load_dem(str(path).encode(), C.byref(nx), C.byref(ny), None, None, None)
        x = np.empty(max(nx.value, 1))
        y = np.empty(max(ny.value, 1))
        z = np.empty(max(nx.value * ny.value, 1))
        self.L.ref_load_dem(str(path).encode(), C.byref(nx), C.byref(ny), _ptr(x), _ptr(y), _ptr(z))
        return x[: nx.value], y[: ny.value], z[: nx.value * ny.value].reshape(ny.value, nx.value)

    for f in (read_binary, export_complex_matrix, export_3d, load_dem):
        setattr(Reference, f.__name__, f)


_ref_files_methods()
