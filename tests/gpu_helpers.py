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
