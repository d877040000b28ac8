"""CPU oracle of the per-peak lightcone state and halo-record packing -- TEST
INFRASTRUCTURE ONLY (the checker of ht_peak_lightcone / ht_pack_halos; never called by the
library).

A scalar restatement, in the reference's operation order and in IEEE FP64 (Python floats)
with Float32 roundings where the reference converts, of:

* Cosmology.chi_to_z and peak_redshift (src/Cosmology/Cosmology.jl:354-385),
* PeakCandidate positions (ext/CUDAExt.jl:3039-3046),
* _hunt, _lagrint_2col and Dlinear_ab's D(a) (Cosmology.jl:97-132, 286-306),
* omega_m_a (Cosmology.jl:52),
* the lightcone loop before the collapse (src/MultiResolution.jl:1097-1130) and the record
  loop after it (MultiResolution.jl:1159-1219) with the field order of HaloRecord /
  ExtHaloRecord (src/IO/Catalog.jl:4-48),
* merge_catalog with lagrangian_exclusion! and volume_reduction! (src/Merger/Merger.jl:38-104,
  src/Merger/Exclusion.jl:81-206) and finalize_eulerian (Merger.jl:114-146); the
  neighbour search is a k-d tree instead of the linked-list hash (both are exhaustive
  within the radius, so the survivors do not depend on it).

fsc_of_z is the C oracle's (RadialShell.jl:181-195).  The cosmology tables themselves are
inputs (built by the host code the reference runs once per run).
"""
from __future__ import annotations

import math

import numpy as np

f32 = np.float32


def cell_centre(c0: float, alatt: float, i: int, n: int) -> float:
    """xbx + alatt (i - cen1), cen1 = 0.5 (n + 1)  (CUDAExt.jl:3039-3046)."""
    cen1 = 0.5 * (n + 1)
    return c0 + alatt * (i - cen1)


def chi_to_z(chis, zs, z_max: float, chi_val: float) -> float:
    """Cosmology.jl:354-371."""
    if chi_val <= chis[0]:
        return 0.0
    if chi_val >= chis[-1]:
        return z_max
    lo, hi = 1, len(zs)                       # 1-based, as the reference
    while hi - lo > 1:
        mid = (lo + hi) >> 1
        if chis[mid - 1] <= chi_val:
            lo = mid
        else:
            hi = mid
    frac = (chi_val - chis[lo - 1]) / (chis[hi - 1] - chis[lo - 1])
    return zs[lo - 1] + frac * (zs[hi - 1] - zs[lo - 1])


def peak_redshift(obs, pos, chis, zs, z_max: float) -> float:
    """Cosmology.jl:376-385."""
    dx = pos[0] - obs[0]
    dy = pos[1] - obs[1]
    dz = pos[2] - obs[2]
    return chi_to_z(chis, zs, z_max, math.sqrt(dx * dx + dy * dy + dz * dz))


def hunt(xx, x: float) -> int:
    """_hunt (Cosmology.jl:117-132): 1-based jlo."""
    n = len(xx)
    ascnd = xx[n - 1] > xx[0]
    jlo, jhi = 0, n + 1
    while jhi - jlo > 1:
        jm = (jhi + jlo) // 2
        if (x > xx[jm - 1]) == ascnd:
            jlo = jm
        else:
            jhi = jm
    return jlo


def growth_D(g, ai: float) -> float:
    """First value of Dlinear_ab (Cosmology.jl:286-306): D(a)/a by 4-point Lagrange
    interpolation (2-point at the ends, _lagrint_2col :97-115), times a.  A 4-point window
    that would start before the first entry starts at it (the reference would index out of
    bounds there, at a ~ 1/1000)."""
    atab, Dtab, ntab = g.atab, g.D_atab, len(g.atab)
    if g.amintab < ai < g.amaxtab:
        kk = hunt(atab, ai)
        if kk < 2 or kk >= ntab:
            nlint, kkl = 2, max(kk - 1, 1)
        else:
            nlint, kkl = 4, max(kk - 2, 1)
        xa = [float(atab[kkl - 1 + q]) for q in range(nlint)]
        va = [float(Dtab[kkl - 1 + q]) for q in range(nlint)]
        x = ai
        if nlint == 4:
            def coef(i, a_, b_, c_):
                return (x - xa[a_]) / (xa[i] - xa[a_]) * (x - xa[b_]) / (xa[i] - xa[b_]) * \
                    (x - xa[c_]) / (xa[i] - xa[c_])
            a1, a2, a3, a4 = coef(0, 1, 2, 3), coef(1, 0, 2, 3), coef(2, 0, 1, 3), coef(3, 0, 1, 2)
            p = a1 * va[0] + a2 * va[1] + a3 * va[2] + a4 * va[3]
        else:
            a1 = (x - xa[1]) / (xa[0] - xa[1])
            a2 = 1.0 - a1
            p = a1 * va[0] + a2 * va[1]
        return p * ai
    if ai >= g.amaxtab:
        return g.D_a0 * ai
    return g.D_ainfty * ai


def omega_m_a(Om: float, OL: float, a: float) -> float:
    a3 = a * a * a
    return (Om / a3) / (Om / a3 + OL)


def lightcone(i, j, k, n: int, centre, alatt: float, obs, chis, zs, zmax_tab: float,
              z_max: float, fsc_of_z):
    """MultiResolution.jl:1097-1130 per peak: (z Float64, ZZon Float32, fcrit Float32,
    kept 0-based indices)."""
    npk = len(i)
    z = np.zeros(npk)
    zz = np.zeros(npk, np.float32)
    fc = np.zeros(npk, np.float32)
    for p in range(npk):
        pos = (cell_centre(centre[0], alatt, int(i[p]), n),
               cell_centre(centre[1], alatt, int(j[p]), n),
               cell_centre(centre[2], alatt, int(k[p]), n))
        z[p] = peak_redshift(obs, pos, chis, zs, zmax_tab)
        zz[p] = f32(1.0 + z[p])
        fc[p] = f32(fsc_of_z(z[p]))
    return z, zz, fc, np.nonzero(z <= z_max)[0]


def halo_records(peaks: dict, res: dict, n: int, centre, alatt: float, growth, Om: float,
                 OL: float, *, ZZon: float = 1.0, z_max: float = math.inf, ilpt: int = 2,
                 ioutshear: int = 0) -> np.ndarray:
    """MultiResolution.jl:1159-1219: records of the peaks with RTHL > 0 (and z <= z_max on
    a lightcone) in peak order; 11 fields, or 33 when ioutshear >= 1 (Catalog.jl:4-48).
    peaks: i, j, k, Rf, FcRf, d2Rf (or None), z (or None); res: the 14 result arrays
    (Sbar etc. as (npeaks, 3) rows, strain as 9 column-major values per peak)."""
    rows = []
    R = lambda name: np.asarray(res[name], np.float32)
    RTHL, Fbarx = R("RTHL"), R("Fbarx")
    Sbar, Sbar2 = R("Sbar").reshape(-1, 3), R("Sbar2").reshape(-1, 3)
    zarr = peaks.get("z")
    for p in range(len(peaks["i"])):
        if RTHL[p] <= 0:
            continue
        ZZon_pk = ZZon
        if zarr is not None:
            z_pk = float(zarr[p])
            ZZon_pk = 1.0 + z_pk
            if z_pk > z_max:
                continue
        a_pk = 1.0 / ZZon_pk
        D_pk = growth_D(growth, a_pk)
        D32 = f32(D_pk)
        x = cell_centre(centre[0], alatt, int(peaks["i"][p]), n)
        y = cell_centre(centre[1], alatt, int(peaks["j"][p]), n)
        zc = cell_centre(centre[2], alatt, int(peaks["k"][p]), n)
        rec = [f32(x), f32(y), f32(zc), Sbar[p, 0] * D32, Sbar[p, 1] * D32, Sbar[p, 2] * D32,
               f32(float(RTHL[p]) * alatt)]
        if ilpt >= 2:
            # coef2_base * Om_a^(-1/143) * D_pk^2: the square first, then left to right
            coef = f32(-3.0 / 7.0 * omega_m_a(Om, OL, a_pk) ** (-1.0 / 143) * (D_pk * D_pk))
            rec += [Sbar2[p, 0] * coef, Sbar2[p, 1] * coef, Sbar2[p, 2] * coef]
        else:
            rec += [f32(0), f32(0), f32(0)]
        rec.append(Fbarx[p])
        if ioutshear >= 1:
            st = R("strain").reshape(-1, 9)[p]          # (L, K) at L + 3 K
            g3 = lambda nm: list(R(nm).reshape(-1, 3)[p])
            d2 = peaks.get("d2Rf")
            rec += [R("e_v")[p], R("p_v")[p], st[0], st[4], st[8], st[7], st[6], st[3],
                    R("d2F")[p], R("zvir_half")[p]] + g3("gradpk") + g3("gradpkf") + \
                [f32(float(peaks["Rf"][p])), f32(peaks["FcRf"][p]),
                 f32(d2[p]) if d2 is not None else f32(0)] + g3("gradpkrf")
        rows.append(np.array(rec, np.float32))
    width = 33 if ioutshear >= 1 else 11
    return np.array(rows, np.float32).reshape(-1, width)


def growth_f(g, ai: float) -> float:
    """Second value of Dlinear_ab: dlnD/dlna with the same Lagrange weights."""
    atab, ftab, ntab = g.atab, g.dlnD_dlnatab, len(g.atab)
    if g.amintab < ai < g.amaxtab:
        kk = hunt(atab, ai)
        if kk < 2 or kk >= ntab:
            nlint, kkl = 2, max(kk - 1, 1)
        else:
            nlint, kkl = 4, max(kk - 2, 1)
        xa = [float(atab[kkl - 1 + q]) for q in range(nlint)]
        va = [float(ftab[kkl - 1 + q]) for q in range(nlint)]
        x = ai
        if nlint == 4:
            def coef(i, a_, b_, c_):
                return (x - xa[a_]) / (xa[i] - xa[a_]) * (x - xa[b_]) / (xa[i] - xa[b_]) * \
                    (x - xa[c_]) / (xa[i] - xa[c_])
            a1, a2, a3, a4 = coef(0, 1, 2, 3), coef(1, 0, 2, 3), coef(2, 0, 1, 3), coef(3, 0, 1, 2)
            return a1 * va[0] + a2 * va[1] + a3 * va[2] + a4 * va[3]
        a1 = (x - xa[1]) / (xa[0] - xa[1])
        return a1 * va[0] + (1.0 - a1) * va[1]
    return g.HD_Ha0 if ai >= g.amaxtab else g.HD_Hainfty


def sphere_overlap(d: float, r1: float, r2: float):
    """Exclusion.jl:81-97."""
    if d >= r1 + r2 or d <= abs(r1 - r2):
        return 0.0, 0.0
    h1 = (r2 - r1 + d) * (r2 + r1 - d) / (2.0 * d)
    h2 = (r1 - r2 + d) * (r1 + r2 - d) / (2.0 * d)
    return (math.pi / 3.0) * (h1 * h1) * (3.0 * r1 - h1), (math.pi / 3.0) * (h2 * h2) * (3.0 * r2 - h2)


def merge_catalog(rec, volume_reduction: bool = False, fortran_ties: bool = False):
    """Merger.jl:38-104: survivors (input order) with their RTHL, as Float32 rows."""
    from scipy.spatial import cKDTree
    rec = np.asarray(rec, np.float32)
    n = rec.shape[0]
    if n == 0:
        return rec.copy()
    x, y, z = (rec[:, c].astype(np.float64) for c in range(3))
    r = rec[:, 6].astype(np.float64)
    xl, yl, zl, rl = x.tolist(), y.tolist(), z.tolist(), r.tolist()
    order = sorted(range(n), key=lambda i: (-rl[i], xl[i], yl[i], zl[i]))
    tree = cKDTree(np.stack([x, y, z], 1))
    surv = [True] * n

    def dist(i, j):
        dx, dy, dz = xl[j] - xl[i], yl[j] - yl[i], zl[j] - zl[i]
        return math.sqrt(dx * dx + dy * dy + dz * dz)

    for i in order:                              # lagrangian_exclusion! (Exclusion.jl:99-140)
        if not surv[i]:
            continue
        ri = rl[i]
        for j in tree.query_ball_point((xl[i], yl[i], zl[i]), ri * (1 + 1e-9) + 1e-9):
            if j != i and surv[j] and ri >= rl[j] and dist(i, j) < ri:
                surv[j] = False
    new_r = list(rl)
    if volume_reduction:                         # volume_reduction! (Exclusion.jl:152-206)
        rank = [0] * n
        for k, i in enumerate(order):
            rank[i] = k
        dV = [0.0] * n
        for i in order:
            if not surv[i]:
                continue
            ri = rl[i]
            for j in tree.query_ball_point((xl[i], yl[i], zl[i]), 2 * ri * (1 + 1e-9) + 1e-9):
                if j != i and surv[j] and rank[j] > rank[i]:
                    rj = rl[j]
                    d = dist(i, j)
                    if d < ri + rj:
                        v1, v2 = sphere_overlap(d, ri, rj)
                        w = 2.0 if (fortran_ties and rj == ri) else 1.0
                        dV[i] += w * v1
                        dV[j] += w * v2
        for i in range(n):
            if not surv[i]:
                continue
            vol = 4 * math.pi / 3 * (rl[i] * rl[i] * rl[i]) - dV[i]
            if vol <= 0.0:
                surv[i], new_r[i] = False, 0.0
            else:
                new_r[i] = math.cbrt(vol * 3 / (4 * math.pi))
    keep = [i for i in range(n) if surv[i]]
    out = rec[keep].copy()
    out[:, 6] = np.array([new_r[i] for i in keep], np.float32)
    return out


def finalize_eulerian(rec, growth, Om: float, OL: float, obs, chis, zs, zmax_tab: float,
                      ievol: int = 1, z_out: float = 0.0):
    """Merger.jl:114-146 on Float32 rows (a copy is returned)."""
    out = np.array(rec, np.float32, copy=True)
    a_snap = 1.0 / (1.0 + z_out)
    for h in range(out.shape[0]):
        q = out[h]
        d1 = [float(q[3]), float(q[4]), float(q[5])]
        d2 = [float(q[7]), float(q[8]), float(q[9])]
        e = [float(q[c]) + d1[c] + d2[c] for c in range(3)]
        a = a_snap
        if ievol == 1:
            dx, dy, dz = e[0] - obs[0], e[1] - obs[1], e[2] - obs[2]
            rr = math.sqrt(dx * dx + dy * dy + dz * dz)
            a = 1.0 / (1.0 + chi_to_z(chis, zs, zmax_tab, rr)) if rr > 0 else 1.0
        E = math.sqrt(Om * a ** -3 + OL)
        vfac = a * 100.0 * E * growth_f(growth, a)
        q[0:3] = np.array(e, np.float32)
        q[3:6] = np.array([vfac * (d1[c] + 2 * d2[c]) for c in range(3)], np.float32)
        q[7:10] = 0.0
    return out
