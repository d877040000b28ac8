"""Precision study on the small periodic-box workload (128^3 box, L = 250 Mpc/h, 36-cell
wrap, 30 top-hat filters R = 2-40 Mpc/h, nhunt 35): the device path (FP32 fields,
per-lane FP64 shell sums with exact FP64 products, lanes combined in FP64 in a fixed
order, FP64 profile recurrence, eigen solve and barrier interpolation) against the CPU
oracle, which accumulates every sum in FP64 from the same FP32 fields in cell order
(RadialShell.jl:362-446 semantics).  The remaining differences are summation order and
the FP32 rounding of the outputs.

Stated tolerance: on peaks whose collapse decision agrees, RTHL, Fbarx (the catalog
overdensity) and e_v agree to 1e-5 relative (e_v with a 1e-4 absolute floor), and p_v to
1e-5 relative with a 1e-3 absolute floor: p_v = (l3 + l1 - 2 l2) / (2 trace) cancels
eigenvalues of order e_v, and on the most ill-conditioned peaks of this workload (p_v
near 1e-4 with strain traces 100x smaller than the entries) the two FP64 implementations
differ by up to 2.2e-9 in p_v, far below the FP32 catalog resolution of the eigenvalues.
Collapse flips (a peak whose barrier crossing sits within round-off of ZZon) are counted
and must stay below 0.2 % of the peaks.  Run with `-s` to print the error table."""
import os
import time

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from gpu_helpers import SCALAR, VECTOR

pytestmark = pytest.mark.gpu

N, L, NBUFF, NF, RMIN, RMAX, SEED = 128, 250.0, 36, 30, 2.0, 40.0, 12345
SAMPLE = 50000   # every peak of the workload (about 43,000)


def _workload(ht):
    from huntian_b200 import synth
    dev = torch.device("cuda", 0)
    cosmo = synth.Cosmology()
    dk = synth.gaussian_box(N, L, SEED, cosmo, dev)
    psi1, psi2 = synth.displacements(dk, N, L, ilpt=2)
    tile = {"delta": synth.wrap_pad(synth._irfft(dk, N), NBUFF)}
    for nm, t in zip(("etax", "etay", "etaz", "eta2x", "eta2y", "eta2z"), psi1 + psi2):
        tile[nm] = synth.wrap_pad(t, NBUFF)
    nt = N + 2 * NBUFF
    alatt = L / N
    filters = ht.log_filterbank(NF, RMIN, RMAX)
    tab, axes = ht.read_homeltab(os.path.join(GOLDEN, "HomelTab_julia.dat"))
    finder = ht.HaloFinder(ht.nhunt_of(filters[0][2], alatt, NBUFF), tab, *axes)
    fcrit = float(np.float32(finder.fsc_of_z(0.0)))
    mask = torch.zeros((nt,) * 3, dtype=torch.int8, device=dev)
    peaks = ht.HaloFinder.alloc_peaks(1 << 20, dev, False)
    delta_k = torch.fft.rfftn(tile["delta"], dim=(0, 1, 2)).contiguous()
    ds = torch.empty((nt,) * 3, dtype=torch.float32, device=dev)
    for fi, flt in enumerate(filters, start=1):
        finder.smooth_tile(delta_k, nt, nt * alatt, flt[2], 1, out=ds)
        finder.peakfind_filter(ds, mask, NBUFF, fcrit, fi, 1 << 20, peaks)
    torch.cuda.synchronize()
    npk = int(peaks["count"].item())
    return tile, finder, peaks, npk, filters, alatt, fcrit, (tab, axes)


def test_precision_vs_fp64_oracle(ht, oracle):
    tile, finder, peaks, npk, filters, alatt, fcrit, (tab, axes) = _workload(ht)
    assert npk > 5000
    t = tile
    finder.bind_fields(t["delta"], t["etax"], t["etay"], t["etaz"], t["eta2x"], t["eta2y"],
                       t["eta2z"], None)
    fidx = peaks["filter_idx"][:npk].long() - 1
    Rf_all = torch.tensor([f[2] for f in filters], dtype=torch.float64, device="cuda")
    ir2_all = torch.tensor([ht.ir2min_of(f[2], alatt) for f in filters], dtype=torch.int32,
                           device="cuda")
    zz = torch.ones(npk, dtype=torch.float32, device="cuda")
    fc = torch.full((npk,), fcrit, dtype=torch.float32, device="cuda")
    res = finder.analyse(peaks["i"][:npk], peaks["j"][:npk], peaks["k"][:npk], Rf_all[fidx],
                         ir2_all[fidx], zz, fc, alatt, nbuff=NBUFF)
    torch.cuda.synchronize()

    rng = np.random.default_rng(0)
    sel = np.sort(rng.choice(npk, size=min(SAMPLE, npk), replace=False))
    host = {k: v.cpu().numpy() for k, v in t.items()}
    F = oracle.Fields(host["delta"], host["etax"], host["etay"], host["etaz"], host["eta2x"],
                      host["eta2y"], host["eta2z"])
    ct = oracle.CollapseTable(tab, *axes)
    pi, pj, pk = (peaks[c][:npk].cpu().numpy()[sel] for c in ("i", "j", "k"))
    fi = fidx.cpu().numpy()[sel]
    t0 = time.perf_counter()
    o, _ = oracle.analyse_batch(F, pi, pj, pk, ir2_all.cpu().numpy()[fi],
                                Rf_all.cpu().numpy()[fi], 1.0, np.float32(fcrit), alatt, ct,
                                oracle.precompute_shells(finder.nhunt), nbuff=NBUFF,
                                kind="cudakernel")
    t_cpu = time.perf_counter() - t0
    g = {k: v.cpu().numpy() for k, v in res.items()}
    width = ht.RESULT_WIDTH
    gs = {k: (g[k][:npk * width.get(k, 1)].reshape(npk, -1)[sel]) for k in SCALAR + VECTOR}

    gc = gs["RTHL"][:, 0] > 0
    oc = o["RTHL"] > 0
    flips = int((gc != oc).sum())
    both = gc & oc
    floor = {"e_v": 1e-4, "p_v": 1e-3}
    table = []
    worst = {}
    for f in SCALAR + VECTOR:
        gv = gs[f][both].astype(np.float64)
        ov = np.asarray(o[f][both], np.float64).reshape(gv.shape)
        ok = ~(np.isnan(gv).any(1) | np.isnan(ov).any(1))
        scale = np.maximum(np.abs(ov[ok]).max(1), floor.get(f, 1e-6))
        err = np.abs(gv[ok] - ov[ok]).max(1) / scale
        worst[f] = float(err.max()) if err.size else 0.0
        table.append((f, worst[f], float(np.median(err)) if err.size else 0.0))
    print(f"\nprecision: {len(sel)} of {npk} peaks, {int(both.sum())} collapsed in both, "
          f"{flips} flips, oracle {t_cpu:.1f} s")
    print(f"{'field':10s} {'max rel err':>12s} {'median':>12s}")
    for f, mx, med in table:
        print(f"{f:10s} {mx:12.3e} {med:12.3e}")
    assert flips <= max(1, int(0.002 * len(sel)))
    for f in ("RTHL", "Fbarx", "e_v", "p_v"):
        assert worst[f] <= 1e-5, (f, worst[f])
