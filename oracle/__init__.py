"""CPU oracle for the halo-finding hot path -- TEST INFRASTRUCTURE ONLY.

A plain-C FP64 restatement of the reference (guanyilun/Huntian.jl) peak finder and
radial-shell collapse, loaded with ctypes.  Only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline leg use it, as the checker; the CUDA library never links
or calls it.

Array convention: 3-D fields are numpy arrays of shape (n3, n2, n1) in C order, which is
byte-for-byte Julia's column-major (n1, n2, n3) array; cell (i, j, k) (1-based) is
``a[k-1, j-1, i-1]``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")


def build(force: bool = False) -> str:
    """Compile liboracle.so with the Makefile beside this file."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < max(os.path.getmtime(os.path.join(_HERE, f))
                                           for f in ("ht_oracle.c", "or_collapse.c", "ht_oracle.h"))):
        subprocess.run(["make", "-s", "-C", _HERE, "-B", "liboracle.so"], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


class Cell(C.Structure):
    _fields_ = [("di", C.c_int32), ("dj", C.c_int32), ("dk", C.c_int32), ("r2", C.c_int32)]


class CTab(C.Structure):
    _fields_ = [("table", C.POINTER(C.c_float)), ("nx", C.c_int), ("ny", C.c_int),
                ("nz", C.c_int), ("x1", C.c_double), ("x2", C.c_double), ("y1", C.c_double),
                ("y2", C.c_double), ("z1", C.c_double), ("z2", C.c_double),
                ("out_val", C.c_double)]


class Grid(C.Structure):
    _fields_ = [("delta", C.c_void_p), ("etax", C.c_void_p), ("etay", C.c_void_p),
                ("etaz", C.c_void_p), ("eta2x", C.c_void_p), ("eta2y", C.c_void_p),
                ("eta2z", C.c_void_p), ("mask", C.c_void_p), ("lapd", C.c_void_p),
                ("n1", C.c_int), ("n2", C.c_int), ("n3", C.c_int)]


RESULT_FIELDS = [("RTHL", 1), ("Srb", 1), ("Sbar", 3), ("Sbar2", 3), ("strain", 9),
                 ("gradpk", 3), ("gradpkrf", 3), ("Fbarx", 1), ("e_v", 1), ("p_v", 1),
                 ("zvir_half", 1), ("gradpkf", 3), ("d2F", 1), ("eigs", 3),
                 # diagnostic: smallest |Fbar - fcrit| / |zvir - ZZon| of the decisions
                 ("margin", 1)]
RESULT_DTYPE = np.dtype([(n, np.float64) if k == 1 else (n, np.float64, (k,))
                         for n, k in RESULT_FIELDS])

_P = C.c_void_p


def _declare(L):
    L.or_precompute_shells.restype = C.c_int64
    L.or_precompute_shells.argtypes = [C.c_int, _P, C.c_int64]
    L.or_hRinteg.restype = C.c_double
    L.or_hRinteg.argtypes = [C.c_double, C.c_double]
    L.or_atab4.argtypes = [_P]
    L.or_interp.restype = C.c_double
    L.or_interp.argtypes = [C.POINTER(CTab), C.c_double, C.c_double, C.c_double]
    L.or_fsc_of_z.restype = C.c_double
    L.or_fsc_of_z.argtypes = [C.c_double, C.POINTER(CTab)]
    L.or_eigvals_sym3.argtypes = [_P, _P]
    L.or_find_peaks.restype = C.c_int64
    L.or_find_peaks.argtypes = [_P, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                C.c_int64, _P, _P, _P, _P]
    L.or_analyse_peak.restype = C.c_int
    L.or_analyse_peak.argtypes = [C.POINTER(Grid), C.c_int64, C.c_double, C.c_int,
                                  C.c_double, C.c_double, C.POINTER(CTab), _P, C.c_int64,
                                  C.c_int, C.c_double, C.c_double, _P]
    L.or_analyse_peak_gpu.restype = C.c_int
    L.or_analyse_peak_gpu.argtypes = [C.POINTER(Grid), C.c_int64, C.c_double, C.c_int,
                                      C.c_double, C.c_double, C.POINTER(CTab), _P,
                                      C.c_int64, C.c_int, C.c_double, C.c_double, C.c_int, _P]
    L.or_analyse_batch.argtypes = [C.POINTER(Grid), C.c_int64, _P, _P, _P, _P, _P, _P, _P,
                                   C.c_double, C.POINTER(CTab), _P, C.c_int64, C.c_int,
                                   C.c_double, C.c_int, _P, _P, C.c_int]
    L.or_max_threads.restype = C.c_int
    L.or_set_exact_products.argtypes = [C.c_int]


def _ptr(a):
    return None if a is None else a.ctypes.data


def precompute_shells(rmax: int) -> np.ndarray:
    """RadialShell.precompute_shells: (N, 4) int32 rows (di, dj, dk, r2), sorted by r2."""
    n = lib().or_precompute_shells(rmax, None, 0)
    out = np.zeros((n, 4), dtype=np.int32)
    lib().or_precompute_shells(rmax, out.ctypes.data, n)
    return out


def build_shell_tables(cells: np.ndarray):
    """ShellAnalysisGPU.build_shell_tables: (start (0-based), count, r2) per shell."""
    r2 = cells[:, 3]
    edges = np.flatnonzero(np.diff(r2)) + 1
    start = np.concatenate([[0], edges]).astype(np.int64)
    count = np.diff(np.concatenate([start, [len(r2)]])).astype(np.int32)
    return start, count, r2[start].astype(np.int32)


def hRinteg(u0: float, u12: float) -> float:
    return lib().or_hRinteg(u0, u12)


def atab4() -> np.ndarray:
    out = np.zeros(1101)
    lib().or_atab4(out.ctypes.data)
    return out


class CollapseTable:
    """Collapse table: Float32 (nx, ny, nz) column-major values + axes, -1 outside."""

    def __init__(self, table, X1, X2, Y1, Y2, Z1, Z2, out_val=-1.0):
        t = np.asarray(table, dtype=np.float32)
        if t.ndim == 3:
            # given as a (nz, ny, nx) C-ordered array (Julia column-major bytes)
            self.nz, self.ny, self.nx = t.shape
        else:
            raise ValueError("table must be 3-D")
        self.table = np.ascontiguousarray(t)
        self.axes = tuple(float(v) for v in (X1, X2, Y1, Y2, Z1, Z2))
        self.out_val = float(out_val)
        self._c = CTab(self.table.ctypes.data_as(C.POINTER(C.c_float)), self.nx, self.ny,
                       self.nz, *self.axes, self.out_val)

    @property
    def c(self):
        return C.byref(self._c)

    def __call__(self, x, y, z) -> float:
        return lib().or_interp(self.c, float(x), float(y), float(z))

    def fsc_of_z(self, z: float) -> float:
        return lib().or_fsc_of_z(float(z), self.c)


def read_homeltab(path: str) -> CollapseTable:
    """CollapseTable.read_homeltab: 3 x Int32 + 6 x Float32 header, Float32 table."""
    raw = open(path, "rb").read()
    nx, ny, nz = np.frombuffer(raw[:12], dtype="<i4")
    ax = np.frombuffer(raw[12:36], dtype="<f4").astype(np.float64)
    tab = np.frombuffer(raw[36:36 + 4 * nx * ny * nz], dtype="<f4").reshape(nz, ny, nx)
    return CollapseTable(tab, *ax)


def eigvals_sym3(a) -> np.ndarray:
    a = np.asarray(a, dtype=np.float64)
    buf = np.ascontiguousarray(a.T).reshape(9)   # column-major
    lam = np.zeros(3)
    lib().or_eigvals_sym3(buf.ctypes.data, lam.ctypes.data)
    return lam


def find_peaks(delta, mask, nbuff: int, fcrit: float, max_peaks: int = 2_000_000):
    """PeakFind.find_peaks on a (n3, n2, n1) field; mutates mask.  Returns
    (i, j, k, delta) arrays, 1-based, in k/j/i scan order."""
    delta = np.ascontiguousarray(delta, dtype=np.float32)
    assert mask.dtype == np.int8 and mask.flags.c_contiguous and mask.shape == delta.shape
    n3, n2, n1 = delta.shape
    inner = max(0, n1 - 2 * nbuff) * max(0, n2 - 2 * nbuff) * max(0, n3 - 2 * nbuff)
    cap = int(min(max_peaks, max(inner, 1)))
    oi = np.zeros(cap, np.int32); oj = np.zeros(cap, np.int32); ok = np.zeros(cap, np.int32)
    od = np.zeros(cap, np.float32)
    n = lib().or_find_peaks(delta.ctypes.data, mask.ctypes.data, n1, n2, n3, nbuff,
                            float(np.float32(fcrit)), max_peaks, oi.ctypes.data,
                            oj.ctypes.data, ok.ctypes.data, od.ctypes.data)
    return oi[:n].copy(), oj[:n].copy(), ok[:n].copy(), od[:n].copy()


class Fields:
    """A tile of FP32 fields for the oracle (kept alive while the C struct points at it)."""

    def __init__(self, delta, etax, etay, etaz, eta2x=None, eta2y=None, eta2z=None,
                 mask=None, lapd=None):
        def f(a):
            return None if a is None else np.ascontiguousarray(a, dtype=np.float32)
        self.delta, self.etax, self.etay, self.etaz = f(delta), f(etax), f(etay), f(etaz)
        self.eta2x, self.eta2y, self.eta2z = f(eta2x), f(eta2y), f(eta2z)
        self.lapd = f(lapd)
        if mask is not None:
            assert mask.dtype == np.int8 and mask.flags.c_contiguous
        self.mask = mask
        n3, n2, n1 = self.delta.shape
        self._c = Grid(_ptr(self.delta), _ptr(self.etax), _ptr(self.etay), _ptr(self.etaz),
                       _ptr(self.eta2x), _ptr(self.eta2y), _ptr(self.eta2z), _ptr(self.mask),
                       _ptr(self.lapd), n1, n2, n3)

    @property
    def c(self):
        return C.byref(self._c)


KIND = {"radialshell": 0, "shellgpu": 1, "cudakernel": 2}


def analyse_peak(fields: Fields, ipp: int, alatt: float, ir2min: int, ZZon: float,
                 Rfclvi: float, ct: CollapseTable, shells: np.ndarray, *, nbuff: int = 0,
                 rmax2rs: float = 0.0, fcrit_override=None, kind: str = "radialshell"):
    """One peak.  kind: 'radialshell' (RadialShell.analyse_peak), 'shellgpu'
    (ShellAnalysisGPU.analyse_peak_gpu), 'cudakernel' (reference CUDA kernel semantics)."""
    out = np.zeros(1, dtype=RESULT_DTYPE)
    fc = -1.0 if fcrit_override is None else float(fcrit_override)
    cells = np.ascontiguousarray(shells, dtype=np.int32)
    if kind == "radialshell":
        code = lib().or_analyse_peak(fields.c, ipp, alatt, ir2min, ZZon, Rfclvi, ct.c,
                                     cells.ctypes.data, len(cells), nbuff, rmax2rs, fc,
                                     out.ctypes.data)
    else:
        code = lib().or_analyse_peak_gpu(fields.c, ipp, alatt, ir2min, ZZon, Rfclvi, ct.c,
                                         cells.ctypes.data, len(cells), nbuff, rmax2rs, fc,
                                         1 if kind == "cudakernel" else 0, out.ctypes.data)
    return out[0], code


def analyse_batch(fields: Fields, pi, pj, pk, ir2min, Rf, ZZon, fcrit, alatt: float,
                  ct: CollapseTable, shells: np.ndarray, *, nbuff: int = 0,
                  rmax2rs: float = 0.0, kind: str = "cudakernel", nthreads: int = 0,
                  exact_products: bool = False):
    """Many peaks on all host threads.  Per-peak arrays; fcrit < 0 means fsc_of_z.
    exact_products: form every cell product in Float64 (the full-FP64 oracle) instead of
    rounding it to Float32 as the reference does."""
    n = len(pi)
    a32 = lambda v: np.ascontiguousarray(np.broadcast_to(v, (n,)), dtype=np.int32)
    a64 = lambda v: np.ascontiguousarray(np.broadcast_to(v, (n,)), dtype=np.float64)
    pi, pj, pk, ir2 = a32(pi), a32(pj), a32(pk), a32(ir2min)
    Rf, ZZon, fcrit = a64(Rf), a64(ZZon), a64(fcrit)
    out = np.zeros(n, dtype=RESULT_DTYPE)
    codes = np.zeros(n, dtype=np.int32)
    cells = np.ascontiguousarray(shells, dtype=np.int32)
    lib().or_set_exact_products(1 if exact_products else 0)
    lib().or_analyse_batch(fields.c, n, pi.ctypes.data, pj.ctypes.data, pk.ctypes.data,
                           ir2.ctypes.data, Rf.ctypes.data, ZZon.ctypes.data,
                           fcrit.ctypes.data, alatt, ct.c, cells.ctypes.data, len(cells),
                           nbuff, rmax2rs, KIND[kind], out.ctypes.data, codes.ctypes.data,
                           nthreads)
    lib().or_set_exact_products(0)
    return out, codes


def max_threads() -> int:
    return lib().or_max_threads()
