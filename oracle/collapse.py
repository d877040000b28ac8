"""Oracle of the collapse-table generator (test infrastructure): ctypes bindings of
or_collapse.c, the C restatement of the reference's RK4 homogeneous-ellipsoid collapse
(EllipsoidalCollapse.jl:149-590 with solver = :rk4), of its adaptive Tsit5 path
(solver = :diffeq, :333-485) and of the table sweep
(CollapseTable.jl:22-76).  Only the tests and the bench's CPU baseline use it."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib


class Growth(C.Structure):
    _fields_ = [("atab", C.POINTER(C.c_double)), ("D_atab", C.POINTER(C.c_double)),
                ("dlnD", C.POINTER(C.c_double)), ("ntab", C.c_int),
                ("amintab", C.c_double), ("amaxtab", C.c_double),
                ("D_ainfty", C.c_double), ("D_a0", C.c_double),
                ("HD_Hainfty", C.c_double), ("HD_Ha0", C.c_double)]


class Ellipsoid(C.Structure):
    _fields_ = [("Om", C.c_double), ("OL", C.c_double), ("iforce_strat", C.c_int),
                ("ivir_strat", C.c_int), ("fcoll", C.c_double * 3), ("tfac", C.c_double),
                ("nstepmax", C.c_int), ("zinit_fac", C.c_double), ("growth", Growth),
                ("solver", C.c_int)]


def _declare(L):
    if getattr(L, "_collapse_declared", False):
        return
    L.or_dlinear_ab.argtypes = [C.POINTER(Growth), C.c_double, C.POINTER(C.c_double),
                                C.POINTER(C.c_double)]
    L.or_dfnofa.argtypes = [C.POINTER(Growth), C.c_double]
    L.or_dfnofa.restype = C.c_double
    L.or_elliptic_rd.argtypes = [C.c_double] * 3
    L.or_elliptic_rd.restype = C.c_double
    L.or_get_b_2.argtypes = [C.c_double] * 3 + [C.POINTER(C.c_double)]
    L.or_evolve_ellipse.argtypes = [C.POINTER(Ellipsoid), C.c_double, C.c_double, C.c_double,
                                    C.c_int, C.POINTER(C.c_double)]
    L.or_evolve_ellipse.restype = C.c_int
    L.or_pow_pos.argtypes = [C.c_double, C.c_double]
    L.or_pow_pos.restype = C.c_double
    L.or_make_table.argtypes = [C.POINTER(Ellipsoid)] + [C.c_int] * 3 + [C.c_double] * 6 + \
        [C.c_void_p]
    L._collapse_declared = True


def _lib():
    L = lib()
    _declare(L)
    return L


class EllipsoidOracle:
    """An EllipsoidParams (defaults of EllipsoidalCollapse.jl:27-45) over the growth tables
    `g` (anything with the DlinearTables fields) and the cosmology's Om, OL."""

    def __init__(self, g, Om: float, OL: float, iforce_strat: int = 4, ivir_strat: int = 2,
                 fcoll=(0.01, 0.171, 0.171), tfac: float = 0.01, nstepmax: int = 10000,
                 zinit_fac: float = 20.0, solver: str = "rk4"):
        self._keep = [np.ascontiguousarray(g.atab, np.float64),
                      np.ascontiguousarray(g.D_atab, np.float64),
                      np.ascontiguousarray(g.dlnD_dlnatab, np.float64)]
        P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        gr = Growth(P(self._keep[0]), P(self._keep[1]), P(self._keep[2]), len(self._keep[0]),
                    g.amintab, g.amaxtab, g.D_ainfty, g.D_a0, g.HD_Hainfty, g.HD_Ha0)
        if solver not in ("rk4", "diffeq"):
            raise ValueError(f"solver {solver!r}: 'rk4' or 'diffeq'")
        self.s = Ellipsoid(Om, OL, iforce_strat, ivir_strat, (C.c_double * 3)(*fcoll), tfac,
                           nstepmax, zinit_fac, gr, 1 if solver == "diffeq" else 0)

    def dlinear_ab(self, a: float):
        d, h = C.c_double(), C.c_double()
        _lib().or_dlinear_ab(C.byref(self.s.growth), a, C.byref(d), C.byref(h))
        return d.value, h.value

    def dfnofa(self, a: float) -> float:
        return _lib().or_dfnofa(C.byref(self.s.growth), a)

    def evolve(self, Frho: float, e_v: float, p_v: float, idynax: int = 1):
        """(zvir, D, Frho D, steps) of evolve_ellipse_full with this oracle's solver."""
        out = (C.c_double * 3)()
        n = _lib().or_evolve_ellipse(C.byref(self.s), Frho, e_v, p_v, idynax, out)
        return out[0], out[1], out[2], n

    def make_table(self, nx=50, ny=20, nz=20, X1=float(np.log10(1.5)), X2=float(np.log10(8.0)),
                   Y1=0.0, Y2=0.5, Z1=-1.0 + 1e-4, Z2=1.0 - 1e-4) -> np.ndarray:
        """make_table: Float32 (nx, ny, nz), returned as a Fortran-ordered array."""
        t = np.zeros(nx * ny * nz, np.float32)
        _lib().or_make_table(C.byref(self.s), nx, ny, nz, X1, X2, Y1, Y2, Z1, Z2,
                             t.ctypes.data)
        return t.reshape((nx, ny, nz), order="F")


def elliptic_rd(x: float, y: float, z: float) -> float:
    return _lib().or_elliptic_rd(x, y, z)


def get_b_2(a1: float, a2: float, a3: float) -> np.ndarray:
    b = (C.c_double * 3)()
    _lib().or_get_b_2(a1, a2, a3, b)
    return np.array(b[:])
