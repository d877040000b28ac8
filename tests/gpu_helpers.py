"""Shared helpers of the GPU parity tests (run the library on numpy inputs)."""
import numpy as np
import torch


def to_dev(a, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def gpu_find_peaks(ht, finder, fields_s, mask, nbuff, fcrits, max_peaks=1 << 20, lapd_s=None):
    """Run the library's peak scan over several smoothed fields (mask carried)."""
    mask_d = to_dev(mask, torch.int8)
    out = ht.HaloFinder.alloc_peaks(max_peaks, "cuda", lapd_s is not None)
    for fi, (ds, fc) in enumerate(zip(fields_s, fcrits), start=1):
        ls = to_dev(lapd_s[fi - 1]) if lapd_s is not None else None
        finder.peakfind_filter(to_dev(ds), mask_d, nbuff, fc, fi, max_peaks, out, lapd_s=ls)
    torch.cuda.synchronize()
    n = int(out["count"].item())
    res = {k: v[:n].cpu().numpy() for k, v in out.items()
           if v is not None and k not in ("count", "found")}
    res["found"] = int(out["found"].item())
    return res, mask_d.cpu().numpy()


def run_shell(finder, fields, peaks, alatt, *, Rf, ir2min, ZZon, fcrit, nbuff=0, mask=None,
              conv="gpu", mode="batched", order=None, diagnostics=False):
    """fields: dict of numpy (n,n,n) arrays (delta, etax.., eta2x.., lapd optional);
    peaks: (i, j, k) 1-based arrays.  Returns dict of numpy results and the mask."""
    dev = {k: (to_dev(v) if v is not None else None) for k, v in fields.items()}
    finder.bind_fields(dev["delta"], dev["etax"], dev["etay"], dev["etaz"], dev.get("eta2x"),
                       dev.get("eta2y"), dev.get("eta2z"), dev.get("lapd"))
    npk = len(peaks[0])
    b = lambda v, dt: to_dev(np.broadcast_to(np.asarray(v), (npk,)), dt)
    mask_d = to_dev(mask, torch.int8) if mask is not None else None
    out = finder.alloc_results(npk, "cuda", diagnostics=diagnostics)
    for k, v in out.items():   # poison: every entry must be written by the call
        v.fill_(float("nan") if v.is_floating_point() else -7)
    order_d = to_dev(order, torch.int32) if order is not None else None
    out = finder.analyse(b(peaks[0], torch.int32), b(peaks[1], torch.int32),
                         b(peaks[2], torch.int32), b(Rf, torch.float64),
                         b(ir2min, torch.int32), b(ZZon, torch.float32),
                         b(fcrit, torch.float32), alatt, nbuff=nbuff, mask=mask_d,
                         conv=conv, mode=mode, out=out, order=order_d)
    torch.cuda.synchronize()
    res = {k: v.cpu().numpy() for k, v in out.items()}
    for k in ("strain",):
        res[k] = res[k][:9 * npk].reshape(npk, 9)
    for k in ("eigs", "Sbar", "Sbar2", "gradpk", "gradpkf", "gradpkrf"):
        res[k] = res[k][:3 * npk].reshape(npk, 3)
    for k in ("RTHL", "Fbarx", "e_v", "p_v", "Srb", "d2F", "zvir_half", "walk_shells",
              "collapse_shell"):
        if k in res:
            res[k] = res[k][:npk]
    return res, (mask_d.cpu().numpy() if mask_d is not None else None)


SCALAR = ("RTHL", "Fbarx", "e_v", "p_v", "Srb", "d2F", "zvir_half")
VECTOR = ("Sbar", "Sbar2", "gradpk", "gradpkf", "gradpkrf", "strain", "eigs")


def compare(gpu, ora, rel=1e-5, abs_floor=None):
    """Per-peak comparison of GPU results with oracle results (structured array).
    Returns (list of mismatching peak indices with the worst field, collapse flips)."""
    abs_floor = abs_floor or {}
    npk = len(ora)
    bad, flips = [], []
    for p in range(npk):
        gc, oc = gpu["RTHL"][p] > 0, ora["RTHL"][p] > 0
        if gc != oc:
            flips.append(p)
            continue
        worst = None
        for f in SCALAR + VECTOR:
            g = np.atleast_1d(np.asarray(gpu[f][p], np.float64))
            o = np.atleast_1d(np.asarray(ora[f][p], np.float64))
            if f == "strain":
                o = o.reshape(9)
            if np.isnan(o).any() or np.isnan(g).any():
                if not np.array_equal(np.isnan(o), np.isnan(g)):
                    worst = (f, "nan")
                continue
            scale = np.maximum(np.abs(o).max(initial=0.0), abs_floor.get(f, 1e-6))
            err = np.abs(g - o).max() / scale
            if err > rel:
                worst = (f, float(err))
        if worst:
            bad.append((p, worst))
    return bad, flips


def make_box_workload(ht, n, L, nbuff, nf, rmin, rmax, seed, max_peaks=1 << 23):
    """A periodic-box workload as the benchmark builds it: seeded BBKS Gaussian field with
    2LPT displacements on an n^3 box (library-independent torch code), wrapped to an
    (n + 2 nbuff)^3 tile; nf log-spaced top-hat filters R = rmin..rmax smoothed by the
    library and scanned with the mask carried.  Returns a dict with the device tile, the
    finder, the peaks and the per-peak filter parameters."""
    import os
    from huntian_b200 import synth
    from conftest import GOLDEN
    dev = torch.device("cuda", 0)
    cosmo = synth.Cosmology()
    dk = synth.gaussian_box(n, L, seed, cosmo, dev)
    psi1, psi2 = synth.displacements(dk, n, L, ilpt=2)
    tile = {"delta": synth.wrap_pad(synth._irfft(dk, n), nbuff)}
    for nm, t in zip(("etax", "etay", "etaz", "eta2x", "eta2y", "eta2z"), psi1 + psi2):
        tile[nm] = synth.wrap_pad(t, nbuff)
    del dk, psi1, psi2
    nt = n + 2 * nbuff
    alatt = L / n
    filters = ht.log_filterbank(nf, rmin, rmax)
    tab, axes = ht.read_homeltab(os.path.join(GOLDEN, "HomelTab_julia.dat"))
    finder = ht.HaloFinder(ht.nhunt_of(filters[0][2], alatt, nbuff), tab, *axes)
    fcrit = float(np.float32(finder.fsc_of_z(0.0)))
    mask = torch.zeros((nt,) * 3, dtype=torch.int8, device=dev)
    peaks = ht.HaloFinder.alloc_peaks(max_peaks, dev, False)
    delta_k = torch.fft.rfftn(tile["delta"], dim=(0, 1, 2)).contiguous()
    ds = torch.empty((nt,) * 3, dtype=torch.float32, device=dev)
    for fi, flt in enumerate(filters, start=1):
        finder.smooth_tile(delta_k, nt, nt * alatt, flt[2], 1, out=ds)
        finder.peakfind_filter(ds, mask, nbuff, fcrit, fi, max_peaks, peaks)
    torch.cuda.synchronize()
    del delta_k, ds
    npk = int(peaks["count"].item())
    fidx = peaks["filter_idx"][:npk].long() - 1
    Rf_all = torch.tensor([f[2] for f in filters], dtype=torch.float64, device=dev)
    ir2_all = torch.tensor([ht.ir2min_of(f[2], alatt) for f in filters], dtype=torch.int32,
                           device=dev)
    args = (peaks["i"][:npk], peaks["j"][:npk], peaks["k"][:npk], Rf_all[fidx], ir2_all[fidx],
            torch.ones(npk, dtype=torch.float32, device=dev),
            torch.full((npk,), fcrit, dtype=torch.float32, device=dev), alatt)
    return {"tile": tile, "finder": finder, "peaks": peaks, "npk": npk, "filters": filters,
            "alatt": alatt, "fcrit": fcrit, "tab": tab, "axes": axes, "nbuff": nbuff,
            "fidx": fidx, "Rf_all": Rf_all, "ir2_all": ir2_all, "args": args}


def oracle_sample(oracle, W, sel, kind, exact_products=False, with_codes=False):
    """Oracle results (and its time in seconds) for the peaks `sel` of a workload;
    exact_products: the full-FP64 variant (cell products formed exactly); with_codes: also
    return the per-peak reject codes (0 collapsed, 1 premask, 2 no fcrit crossing,
    3 m0 = 1, 4 no collapse, 5 RTHL <= 0)."""
    import time
    host = {k: v.cpu().numpy() for k, v in W["tile"].items()}
    F = oracle.Fields(host["delta"], host["etax"], host["etay"], host["etaz"], host["eta2x"],
                      host["eta2y"], host["eta2z"])
    ct = oracle.CollapseTable(W["tab"], *W["axes"])
    p = W["peaks"]
    n = W["npk"]
    pi, pj, pk = (p[c][:n].cpu().numpy()[sel] for c in ("i", "j", "k"))
    fi = W["fidx"].cpu().numpy()[sel]
    t0 = time.perf_counter()
    o, codes = oracle.analyse_batch(F, pi, pj, pk, W["ir2_all"].cpu().numpy()[fi],
                                W["Rf_all"].cpu().numpy()[fi], 1.0, np.float32(W["fcrit"]),
                                W["alatt"], ct, oracle.precompute_shells(W["finder"].nhunt),
                                nbuff=W["nbuff"], kind=kind, exact_products=exact_products)
    if with_codes:
        return o, time.perf_counter() - t0, codes
    return o, time.perf_counter() - t0


def result_rows(ht, res, npk, sel):
    """Per-peak rows of the selected peaks from the library's flat result arrays."""
    width = ht.RESULT_WIDTH
    g = {k: v.cpu().numpy() for k, v in res.items()}
    return {k: g[k][:npk * width.get(k, 1)].reshape(npk, -1)[sel] for k in SCALAR + VECTOR}


def print_report(rep, label):
    print(f"\n{label}: {rep['peaks']} peaks, {rep['collapsed']} collapsed in both, "
          f"{rep['flips']} flips ({rep['flips_unexplained']} above the margin), "
          f"{rep['mismatches']} mismatches, {rep['within_reference_noise']} beyond 1e-5 "
          f"within the reference's rounding noise")
    print(f"{'field':10s} {'max rel err':>12s}")
    for f, v in rep["max_rel"].items():
        print(f"{f:10s} {v:12.3e}")
    if rep["flip_list"]:
        print("flips (peak, oracle decision margin):", rep["flip_list"])
    if rep["mismatch_list"]:
        print("mismatches (peak, field, rel err):", rep["mismatch_list"])
