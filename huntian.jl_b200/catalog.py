"""Lightcone state and halo records of a tile, on the device.

Mirrors the host loops that follow the two GPU entry points in the reference tile stage:

* the per-peak lightcone state before the shell collapse (MultiResolution.jl:1097-1130):
  redshift of every peak seen from the observer (Cosmology.peak_redshift), ZZon = 1 + z,
  fcrit = fsc_of_z(z), and the z <= z_max cut (`peak_lightcone`);
* the HaloRecord / ExtHaloRecord rows of the collapsed peaks (MultiResolution.jl:1159-1219,
  src/IO/Catalog.jl:4-48), with the linear growth factor D(a) of each peak's redshift
  (`pack_halos`);
* the .pksc catalog format (Catalog.jl:48-110: `write_pksc`, `read_pksc`);
* the merge step that follows on the catalog: Lagrangian exclusion and volume reduction
  (Merger.merge_catalog) and the Eulerian finalisation (Merger.finalize_eulerian)
  (`merge_halos`, `finalize_eulerian`).

The cosmology tables (chi -> z, Dlinear) are built once per run on the host, as the
reference does (Cosmology.jl:159-283, 341-347), and copied into the library context
(`set_cosmology`); the per-peak work runs in libhuntian_b200.so.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._lib import HtCatalogPeaks, HtCosmo, HtResults, HtTileGeom, RESULT_NAMES, check

HALO_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "RTHL", "vx2", "vy2", "vz2", "overdensity")
EXT_FIELDS = HALO_FIELDS + (
    "e_v", "p_v", "strain_11", "strain_22", "strain_33", "strain_23", "strain_13",
    "strain_12", "d2F", "zform", "grad_x", "grad_y", "grad_z", "gradf_x", "gradf_y",
    "gradf_z", "Rf", "FcollvRf", "d2FRf", "gradrf_x", "gradrf_y", "gradrf_z")


# ------------------------------------------------------------------ cosmology ----
@dataclass(frozen=True)
class CosmologyParams:
    """Cosmology.CosmologyParams (Cosmology.jl:5-12)."""
    Om: float = 0.31
    OB: float = 0.049
    OL: float = 0.69
    h: float = 0.68
    ns: float = 0.965
    s8: float = 0.81


def E2(z: float, c: CosmologyParams) -> float:
    """H^2(z)/H0^2 for flat LambdaCDM without radiation (Cosmology.jl:15)."""
    zp1 = 1 + z
    return c.Om * (zp1 * zp1 * zp1) + c.OL


def chi(z: float, c: CosmologyParams) -> float:
    """Comoving distance in Mpc/h (Cosmology.jl:21-27): (c/100) int_0^z dz'/E(z')."""
    from scipy.integrate import quad
    val, _ = quad(lambda zp: 1.0 / math.sqrt(E2(zp, c)), 0.0, z, epsabs=0.0, epsrel=1e-12,
                  limit=200)
    return (2.998e5 / 100.0) * val


@dataclass
class ChiToZTable:
    """Cosmology.ChiToZTable (Cosmology.jl:332-347)."""
    zs: np.ndarray
    chis: np.ndarray
    z_max: float


def build_chi_to_z(c: CosmologyParams, z_max: float = 10.0, npts: int = 2000) -> ChiToZTable:
    zs = np.linspace(0.0, z_max, npts)
    return ChiToZTable(zs, np.array([chi(float(z), c) for z in zs]), float(z_max))


@dataclass
class DlinearTables:
    """Cosmology.DlinearTables: D(a)/a and dlnD/dlna on a table of a (Cosmology.jl:64-79)."""
    atab: np.ndarray
    D_atab: np.ndarray
    dlnD_dlnatab: np.ndarray
    amintab: float
    amaxtab: float
    D_ainfty: float
    D_a0: float
    HD_Hainfty: float
    HD_Ha0: float


def _deriv_dlin(y, a, h_val, Omnr, Omvac, Omcurv, OmX, OmB):
    """_deriv_Dlin! (Cosmology.jl:136-157) with Omer = Omhdm = Omnrd = 0, no decay."""
    a3 = a * a * a                      # Julia's a^3 (literal power: two products)
    hub = Omnr + Omvac * a3 + Omcurv * a
    d1 = 1.0 / (h_val * math.sqrt(hub / a3))
    fb = y[2]
    q = Omnr + Omvac * a3 + Omcurv * a
    qs = 0.5 / q
    q_val = qs * (Omnr - 2.0 * Omvac * a3)
    fnr = (OmX + OmB) / Omnr
    if OmB != 0.0 and a <= 1.0e-3:
        fnr = OmX / Omnr
    qf = qs * (Omnr * fnr)
    d3 = 3.0 * qf - fb * fb - (1.0 - q_val) * fb
    return np.array([d1, fb, d3, 0.0, d1 / a])


def dlinear_tables(c: CosmologyParams) -> DlinearTables:
    """Dlinear_tables (Cosmology.jl:159-283): RK4 in ln a of the linear-growth ODE from
    a = 1e-7 to a = 2, tabulating D(a)/a and dlnD/dlna for a >= 1/1001, normalised to
    D(a = 1) = 1."""
    Omnr, Omvac = c.Om, c.OL
    Omcurv = 1.0 - c.Om - c.OL
    OmX = c.Om - c.OB
    amaxtab, amintab_target, ainit, nmax = 1.0 / 0.5, 1.0 / 1001.0, 1.0e-7, 2000
    a = ainit
    alogn = math.log(ainit)
    hh = (math.log(amaxtab) - alogn) / nmax
    t0 = 1.0 / c.h / math.sqrt(Omnr)
    yaeq, yaeq0 = math.sqrt(a), 0.0
    y = np.array([t0 * (2.0 / 3.0 * (yaeq * yaeq * yaeq - yaeq0 * yaeq0 * yaeq0)), math.log(a),
                  0.25 * (math.sqrt(24.0 * OmX / Omnr + 1.0) - 1.0), 0.0,
                  t0 * 2.0 * (yaeq - yaeq0)])
    args = (c.h, Omnr, Omvac, Omcurv, OmX, c.OB)
    atab, Dtab, ftab = [], [], []
    lnorm, bnorm, ip0 = True, 1.0, 0
    for _ in range(nmax):
        w1 = _deriv_dlin(y, a, *args)
        a_half = math.exp(alogn + hh * 0.5)
        w2 = _deriv_dlin(y + hh * w1 * 0.5, a_half, *args)
        w3 = _deriv_dlin(y + hh * w2 * 0.5, a_half, *args)
        alogn = alogn + hh
        a = math.exp(alogn)
        w4 = _deriv_dlin(y + hh * w3, a, *args)
        y = y + hh / 6.0 * (w1 + w4 + 2.0 * (w2 + w3))
        if lnorm and a >= 0.001:
            lnorm = False
            bnorm = math.exp(y[1]) / a
        if amintab_target <= a <= amaxtab:
            atab.append(a)
            Dtab.append(math.exp(y[1]) / a)
            ftab.append(y[2])
            if a >= 1.0 and ip0 == 0:
                ip0 = len(atab)
    atab, Dtab, ftab = np.array(atab), np.array(Dtab), np.array(ftab)
    if ip0 > 1:
        ai = (atab[ip0 - 1] - 1.0) / (atab[ip0 - 1] - atab[ip0 - 2])
        D_agrowth = (Dtab[ip0 - 1] * (1.0 - ai) + Dtab[ip0 - 2] * ai) / bnorm
        fac = 1.0 / (D_agrowth * bnorm)
    else:
        fac = 1.0 / bnorm
    Dtab = Dtab * fac
    return DlinearTables(atab, Dtab, ftab, float(atab[0]), float(atab[-1]), float(Dtab[0]),
                         float(Dtab[-1]), float(ftab[0]), float(ftab[-1]))


def omega_m_a(Om: float, OL: float, a: float) -> float:
    """(Om/a^3)/(Om/a^3 + OL) (Cosmology.jl:52)."""
    a3 = a * a * a
    return (Om / a3) / (Om / a3 + OL)


# ------------------------------------------------------------- library calls ----
def _ptr(t: Optional[torch.Tensor]):
    return None if t is None else t.data_ptr()


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def set_cosmology(finder, cosmo: CosmologyParams, chi2z: ChiToZTable,
                  growth: DlinearTables) -> None:
    """ht_ctx_set_cosmo: copy the run's chi -> z and Dlinear tables into the context."""
    arrs = [np.ascontiguousarray(a, np.float64) for a in
            (chi2z.chis, chi2z.zs, growth.atab, growth.D_atab, growth.dlnD_dlnatab)]
    c = HtCosmo(arrs[0].ctypes.data, arrs[1].ctypes.data, len(arrs[0]), chi2z.z_max,
                arrs[2].ctypes.data, arrs[3].ctypes.data, arrs[4].ctypes.data, len(arrs[2]),
                growth.amintab, growth.amaxtab, growth.D_ainfty, growth.D_a0,
                growth.HD_Hainfty, growth.HD_Ha0, cosmo.Om, cosmo.OL)
    check(_lib.load().ht_ctx_set_cosmo(finder.handle, C.byref(c)))


def tile_geom(n: int, centre, alatt: float) -> HtTileGeom:
    return HtTileGeom(int(n), float(centre[0]), float(centre[1]), float(centre[2]),
                      float(alatt))


def peak_lightcone(finder, i: torch.Tensor, j: torch.Tensor, k: torch.Tensor, n: int, centre,
                   alatt: float, obs, z_max: float, stream=None) -> dict:
    """ht_peak_lightcone on the peak scan's 1-based cells: returns device tensors z
    (Float64), ZZon and fcrit (Float32) for every peak, and `keep`, the indices of the
    peaks with z <= z_max in order (MultiResolution.jl:1097-1130)."""
    npk = int(i.numel())
    dev = i.device
    z = torch.empty(npk, dtype=torch.float64, device=dev)
    zz = torch.empty(npk, dtype=torch.float32, device=dev)
    fc = torch.empty(npk, dtype=torch.float32, device=dev)
    keep = torch.empty(max(npk, 1), dtype=torch.int32, device=dev)
    nkeep = torch.zeros(1, dtype=torch.int64, device=dev)
    g = tile_geom(n, centre, alatt)
    o = (C.c_double * 3)(*[float(v) for v in obs])
    check(_lib.load().ht_peak_lightcone(finder.handle, _ptr(i), _ptr(j), _ptr(k), npk,
                                        C.byref(g), C.cast(o, C.c_void_p), float(z_max),
                                        z.data_ptr(), zz.data_ptr(), fc.data_ptr(),
                                        keep.data_ptr(), nkeep.data_ptr(), _stream(stream)))
    nk = int(nkeep.item())
    return {"z": z, "ZZon": zz, "fcrit": fc, "keep": keep[:nk].long()}


def pack_halos(finder, peaks: dict, results: dict, n: int, centre, alatt: float, *,
               ZZon: float = 1.0, z_max: float = math.inf, ilpt: int = 2, ioutshear: int = 0,
               cap: Optional[int] = None, stream=None) -> torch.Tensor:
    """ht_pack_halos: (nhalo, 11) HaloRecord or (nhalo, 33) ExtHaloRecord rows (Float32,
    device) of the collapsed peaks in peak order.  peaks: i, j, k (Int32 1-based), Rf
    (Float64), FcRf (Float32), d2Rf (Float32 or None) and z (Float64 per-peak redshift, or
    None to use ZZon for every peak); results: the analysis outputs for the same peaks.
    cap: at most this many rows are written (default: one per peak)."""
    npk = int(peaks["i"].numel())
    dev = peaks["i"].device
    width = 33 if ioutshear >= 1 else 11
    rows = npk if cap is None else int(cap)
    out = torch.empty((max(rows, 1), width), dtype=torch.float32, device=dev)
    nh = torch.zeros(1, dtype=torch.int64, device=dev)
    cp = HtCatalogPeaks(*[_ptr(peaks.get(f)) for f in ("i", "j", "k", "Rf", "FcRf", "d2Rf",
                                                        "z")], npk)
    r = HtResults(*[_ptr(results.get(nm)) for nm in RESULT_NAMES], None, None)
    g = tile_geom(n, centre, alatt)
    check(_lib.load().ht_pack_halos(finder.handle, C.byref(cp), C.byref(r), C.byref(g),
                                    float(ZZon), float(z_max), int(ilpt), int(ioutshear),
                                    out.data_ptr(), rows, nh.data_ptr(), _stream(stream)))
    return out[:min(int(nh.item()), rows)]


def merge_halos(finder, records: torch.Tensor, *, volume_reduction: bool = False,
                fortran_ties: bool = False, stream=None) -> torch.Tensor:
    """ht_merge_halos (Merger.merge_catalog, Merger.jl:38-104): Lagrangian exclusion (and
    optionally volume reduction) of (nhalo, 11 | 33) Float32 device records; returns the
    survivors in input order with their RTHL (reduced when volume_reduction)."""
    rec = records.contiguous()
    n, width = (int(rec.shape[0]), int(rec.shape[1])) if rec.dim() == 2 else (0, 11)
    out = torch.empty((max(n, 1), width), dtype=torch.float32, device=rec.device)
    nout = torch.zeros(1, dtype=torch.int64, device=rec.device)
    check(_lib.load().ht_merge_halos(finder.handle, rec.data_ptr() if n else None, n, width,
                                     int(bool(volume_reduction)), int(bool(fortran_ties)),
                                     out.data_ptr(), nout.data_ptr(), _stream(stream)))
    return out[:int(nout.item())]


def finalize_eulerian(finder, records: torch.Tensor, obs=(0.0, 0.0, 0.0), *, ievol: int = 1,
                      z_out: float = 0.0, stream=None) -> torch.Tensor:
    """ht_finalize_eulerian (Merger.finalize_eulerian, Merger.jl:114-146), in place on a
    merged raw catalog: Eulerian positions and km/s velocities.  Uses the chi -> z and
    growth tables of set_cosmology (the reference builds its chi table with z_max = 10)."""
    n = int(records.shape[0]) if records.dim() == 2 else 0
    if n == 0:
        return records
    assert records.is_contiguous() and records.dtype == torch.float32
    o = (C.c_double * 3)(*[float(v) for v in obs])
    check(_lib.load().ht_finalize_eulerian(finder.handle, records.data_ptr(), n,
                                           int(records.shape[1]), C.cast(o, C.c_void_p),
                                           int(ievol), float(z_out), _stream(stream)))
    return records


# --------------------------------------------------------------- .pksc files ----
def write_pksc(path: str, records, RTHLmax: float, z_out: float) -> None:
    """Catalog.write_pksc (Catalog.jl:48-96): Int32 Nhalo, Float32 RTHLmax, Float32 z_out,
    then the Float32 rows (11 or 33 fields each)."""
    rec = records.detach().cpu().numpy() if isinstance(records, torch.Tensor) else records
    rec = np.ascontiguousarray(rec, dtype=np.float32)
    with open(path, "wb") as f:
        f.write(np.int32(rec.shape[0] if rec.ndim == 2 else 0).tobytes())
        f.write(np.float32(RTHLmax).tobytes())
        f.write(np.float32(z_out).tobytes())
        f.write(rec.tobytes())


def read_pksc(path: str):
    """Catalog.read_pksc (Catalog.jl:98-130): (records (nhalo, nfields), RTHLmax, z_out);
    the field count follows from the file size."""
    raw = open(path, "rb").read()
    nhalo = int(np.frombuffer(raw, np.int32, 1, 0)[0])
    RTHLmax = float(np.frombuffer(raw, np.float32, 1, 4)[0])
    z_out = float(np.frombuffer(raw, np.float32, 1, 8)[0])
    data = np.frombuffer(raw, np.float32, offset=12)
    nf = data.size // nhalo if nhalo > 0 else len(HALO_FIELDS)
    return data.reshape(nhalo, nf).copy(), RTHLmax, z_out
