"""Collapse-table generation on the device: the host side of ht_evolve_ellipses and
ht_collapse_table, mirroring the reference's EllipsoidalCollapse / CollapseTable API
(src/EllipsoidalCollapse/EllipsoidalCollapse.jl, src/EllipsoidalCollapse/CollapseTable.jl,
bin/generate_table.jl).

Both of the reference's integrators run on the device, one ellipsoid per thread in FP64:
`solver = "diffeq"` (the reference's default, `_evolve_diffeq`, EllipsoidalCollapse.jl:
440-485: adaptive Tsit5 with abstol 1e-8, reltol 1e-6 and OrdinaryDiffEq's step control,
restated from the published method) and `solver = "rk4"` (the fixed-step port of the
Fortran HomogeneousEllipsoid.f90, which reproduces the shipped HomelTab tables).  Tables
come out in this package's HomelTab layout, (nz, ny, nx) float32 holding Julia's
column-major bytes, ready for write_homeltab / HaloFinder.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._lib import HtEllipsoid, HtGrowth, check
from .catalog import CosmologyParams, DlinearTables, dlinear_tables


@dataclass
class EllipsoidParams:
    """EllipsoidParams (EllipsoidalCollapse.jl:10-45) with the Fortran hpkvd defaults."""
    cosmo: CosmologyParams
    iforce_strat: int = 4
    ivir_strat: int = 2
    fcoll_1: float = 0.01
    fcoll_2: float = 0.171
    fcoll_3: float = 0.171
    tfac: float = 0.01
    nstepmax: int = 10000
    zinit_fac: float = 20.0
    iwant_rd: int = 1
    solver: str = "diffeq"
    dlin_tables: Optional[DlinearTables] = field(default=None, repr=False)

    def __post_init__(self):
        if self.solver not in ("rk4", "diffeq"):
            raise ValueError(f"solver {self.solver!r}: 'diffeq' (adaptive Tsit5) or 'rk4' "
                             "(the fixed-step Fortran path), as EllipsoidalCollapse.jl:23")
        if self.iwant_rd != 1:
            raise ValueError("iwant_rd != 1 (Legendre form) is not implemented, as in the "
                             "reference")
        if self.dlin_tables is None:
            self.dlin_tables = dlinear_tables(self.cosmo)

    def _structs(self):
        e = HtEllipsoid(self.cosmo.Om, self.cosmo.OL, self.iforce_strat, self.ivir_strat,
                        (C.c_double * 3)(self.fcoll_1, self.fcoll_2, self.fcoll_3), self.tfac,
                        self.nstepmax, self.zinit_fac,
                        _lib.HT_SOLVER_TSIT5 if self.solver == "diffeq" else _lib.HT_SOLVER_RK4)
        g = self.dlin_tables
        keep = [np.ascontiguousarray(a, np.float64)
                for a in (g.atab, g.D_atab, g.dlnD_dlnatab)]
        gr = HtGrowth(*(a.ctypes.data for a in keep), len(keep[0]), g.amintab, g.amaxtab,
                      g.D_ainfty, g.D_a0, g.HD_Hainfty, g.HD_Ha0)
        return e, gr, keep


@dataclass
class CollapseTableParams:
    """CollapseTableParams (CollapseTable.jl:8-20): zvir(log10 Frho, e_v, p_v/e_v)."""
    Nx: int = 50
    Ny: int = 20
    Nz: int = 20
    X1: float = math.log10(1.5)
    X2: float = math.log10(8.0)
    Y1: float = 0.0
    Y2: float = 0.5
    Z1: float = -1.0 + 1e-4
    Z2: float = 1.0 - 1e-4

    @property
    def axes(self):
        return (self.X1, self.X2, self.Y1, self.Y2, self.Z1, self.Z2)


def evolve_ellipses(Frho, e_v, p_v, ep: EllipsoidParams, idynax: int = 1,
                    device: int = 0, steps: bool = False):
    """evolve_ellipse_full (EllipsoidalCollapse.jl:492-590) for arrays of ellipsoids on the
    device: returns (zvir, D, Frho D) as float64 CUDA tensors (and the steps taken when
    `steps`), -1 where event `idynax` does not happen before a = 2."""
    dev = torch.device("cuda", device)
    F = torch.as_tensor(Frho, dtype=torch.float64, device=dev).reshape(-1).contiguous()
    E = torch.as_tensor(e_v, dtype=torch.float64, device=dev).reshape(-1).contiguous()
    P = torch.as_tensor(p_v, dtype=torch.float64, device=dev).reshape(-1).contiguous()
    if not (F.numel() == E.numel() == P.numel()):
        raise ValueError("Frho, e_v and p_v need the same length")
    n = F.numel()
    z = torch.empty(n, dtype=torch.float64, device=dev)
    D = torch.empty_like(z)
    fc = torch.empty_like(z)
    st = torch.empty(n, dtype=torch.int32, device=dev)
    e, gr, keep = ep._structs()
    stream = torch.cuda.current_stream(dev).cuda_stream
    check(_lib.load().ht_evolve_ellipses(device, C.byref(e), C.byref(gr), n, F.data_ptr(),
                                         E.data_ptr(), P.data_ptr(), idynax, z.data_ptr(),
                                         D.data_ptr(), fc.data_ptr(), st.data_ptr(), stream))
    return (z, D, fc, st) if steps else (z, D, fc)


def evolve_ellipse_full(Frho: float, e_v: float, p_v: float, ep: EllipsoidParams,
                        idynax: int = 1, device: int = 0):
    """One ellipsoid, as the reference's scalar call: (zvir, D, Frho D) as floats."""
    z, D, fc = evolve_ellipses([Frho], [e_v], [p_v], ep, idynax, device)
    return float(z[0]), float(D[0]), float(fc[0])


def make_table(ep: EllipsoidParams, tp: Optional[CollapseTableParams] = None,
               device: int = 0) -> np.ndarray:
    """make_table / make_table_threaded (CollapseTable.jl:29-76) on the device: the
    (nz, ny, nx) float32 table (Julia's column-major bytes)."""
    tp = tp or CollapseTableParams()
    e, gr, keep = ep._structs()
    out = np.zeros(tp.Nx * tp.Ny * tp.Nz, np.float32)
    check(_lib.load().ht_collapse_table(device, C.byref(e), C.byref(gr), tp.Nx, tp.Ny, tp.Nz,
                                        *tp.axes, out.ctypes.data))
    return out.reshape(tp.Nz, tp.Ny, tp.Nx)


def generate_table(path: str, Om: float = 0.315, OB: float = 0.049, OL: float = 0.685,
                   h: float = 0.674, solver: str = "diffeq", device: int = 0) -> np.ndarray:
    """bin/generate_table.jl [--solver diffeq|rk4]: the default 50 x 20 x 20 table for the
    given cosmology, written as a HomelTab file."""
    from .tables import write_homeltab
    cosmo = CosmologyParams(Om=Om, OB=OB, OL=OL, h=h, ns=0.965, s8=0.808)
    tp = CollapseTableParams()
    t = make_table(EllipsoidParams(cosmo, solver=solver), tp, device)
    write_homeltab(path, t, tp.axes)
    return t
