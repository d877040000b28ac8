"""Train the learned walk-length bracket on synthetic tiles and write its weights.

    python huntian.jl_b200/train_bracket.py [--n 512] [--train-seeds 1-8] [--test-seed 9]
                                            [--epochs 6] [--out huntian.jl_b200/bracket_box512.npz]

Each seed is a 512^3 periodic box (L = 1000 Mpc/h, 54-cell wrap, 60 top-hat filters
R = 1.5-60 Mpc/h, the same generator as bench.py): the peaks of all filters are found,
collapsed once with diagnostics, and (features, radius at which the walk stopped) become
training rows.  Training uses the library's own kernels (ht_bracket_grad, ht_bracket_adam).
The test seed reports the pinball loss, the bracket coverage and the collapse time in
BATCHED (spatial order) and LEARNED (predicted order) modes.  Needs a GPU.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _package():
    name = "huntian_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(
        name, os.path.join(HERE, "__init__.py"), submodule_search_locations=[HERE])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def tile_samples(ht, n, L, nbuff, nf, rmin, rmax, seed, device):
    """(finder, batch tensors, features, target radius, peak count) of one synthetic tile."""
    from huntian_b200 import synth
    dk = synth.gaussian_box(n, L, seed, synth.Cosmology(), device)
    psi1, psi2 = synth.displacements(dk, n, L, ilpt=2)
    tile = {"delta": synth.wrap_pad(synth._irfft(dk, n), nbuff)}
    del dk
    for nm, t in zip(("etax", "etay", "etaz", "eta2x", "eta2y", "eta2z"), psi1 + psi2):
        tile[nm] = synth.wrap_pad(t, nbuff)
    del psi1, psi2
    torch.cuda.empty_cache()
    nt = n + 2 * nbuff
    alatt = L / n
    filters = ht.log_filterbank(nf, rmin, rmax)
    tab, axes = ht.read_homeltab(os.path.join(ROOT, "tests", "golden", "HomelTab_julia.dat"))
    finder = ht.HaloFinder(ht.nhunt_of(filters[0][2], alatt, nbuff), tab, *axes,
                           device=device.index or 0)
    fcrit = float(np.float32(finder.fsc_of_z(0.0)))
    mask = torch.zeros((nt,) * 3, dtype=torch.int8, device=device)
    peaks = ht.HaloFinder.alloc_peaks(8_000_000, device, False)
    dkt = torch.fft.rfftn(tile["delta"], dim=(0, 1, 2)).contiguous()
    ds = torch.empty((nt,) * 3, dtype=torch.float32, device=device)
    for fi, flt in enumerate(filters, start=1):
        finder.smooth_tile(dkt, nt, nt * alatt, flt[2], 1, out=ds)
        finder.peakfind_filter(ds, mask, nbuff, fcrit, fi, 8_000_000, peaks)
    del dkt, ds
    npk = int(peaks["count"].item())
    mask.zero_()
    t = tile
    finder.bind_fields(t["delta"], t["etax"], t["etay"], t["etaz"], t["eta2x"], t["eta2y"],
                       t["eta2z"], None)
    fidx = peaks["filter_idx"][:npk].long() - 1
    Rf = torch.tensor([f[2] for f in filters], dtype=torch.float64, device=device)[fidx]
    ir2 = torch.tensor([ht.ir2min_of(f[2], alatt) for f in filters], dtype=torch.int32,
                       device=device)[fidx]
    zz = torch.ones(npk, dtype=torch.float32, device=device)
    fc = torch.full((npk,), fcrit, dtype=torch.float32, device=device)
    batch = dict(pi=peaks["i"][:npk].clone(), pj=peaks["j"][:npk].clone(),
                 pk=peaks["k"][:npk].clone(), Rf=Rf, ir2min=ir2, ZZon=zz, fcrit=fc)
    out = finder.alloc_results(npk, device, diagnostics=True)
    finder.analyse(*batch.values(), alatt, nbuff=nbuff, mask=mask, out=out)
    rad = torch.sqrt(torch.as_tensor(finder.shell_r2(), dtype=torch.float32, device=device))
    target = rad[(out["walk_shells"][:npk].long() - 1).clamp(min=0)]
    F = ht.bracket.features(finder, *batch.values(), alatt,
                            peak_delta=peaks["delta"][:npk].contiguous())
    return dict(finder=finder, batch=batch, F=F, target=target, npk=npk, alatt=alatt,
                nbuff=nbuff, mask=mask, out=out, tile=tile)


def time_walk(ht, s, mode, cost=None, reps=2):
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s["mask"].zero_()
        a.record()
        s["finder"].analyse(*s["batch"].values(), s["alatt"], nbuff=s["nbuff"], mask=s["mask"],
                            out=s["out"], mode=mode, cost=cost)
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return min(ts)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--train-seeds", default="1-8")
    ap.add_argument("--test-seed", type=int, default=9)
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--out", default=os.path.join(HERE, "bracket_box512.npz"))
    args = ap.parse_args()
    ht = _package()
    dev = torch.device("cuda", 0)
    a, b = (int(x) for x in args.train_seeds.split("-"))
    geo = dict(n=args.n, L=1000.0 * args.n / 512, nbuff=54, nf=60, rmin=1.5, rmax=60.0)
    Fs, Ts = [], []
    for seed in range(a, b + 1):
        t0 = time.perf_counter()
        s = tile_samples(ht, seed=seed, device=dev, **geo)
        Fs.append(s["F"].clone())
        Ts.append(s["target"].clone())
        print(f"seed {seed}: {s['npk']} peaks ({time.perf_counter() - t0:.1f} s)", flush=True)
        del s
        torch.cuda.empty_cache()
    F = torch.cat(Fs)
    T = torch.cat(Ts)
    del Fs, Ts
    s = tile_samples(ht, seed=args.test_seed, device=dev, **geo)
    t0 = time.perf_counter()
    model = ht.bracket.train(s["finder"], F, T, epochs=args.epochs, log=print)
    print(f"trained on {F.shape[0]} rows in {time.perf_counter() - t0:.1f} s", flush=True)
    model.save(args.out)
    pred = ht.bracket.predict(s["finder"], model, s["F"])
    tgt = s["target"]
    cover = float(((tgt >= pred[:, 0]) & (tgt <= pred[:, 1])).float().mean())
    corr = float(torch.corrcoef(torch.stack([pred[:, 1], tgt]))[0, 1])
    cost = pred[:, 1].contiguous()
    res = {"train_rows": int(F.shape[0]), "test_peaks": s["npk"], "coverage_10_90": cover,
           "corr_hi_vs_target": corr,
           "walk_ms_batched": time_walk(ht, s, "batched"),
           "walk_ms_learned": time_walk(ht, s, "learned", cost),
           "walk_ms_true_order": time_walk(ht, s, "learned", tgt.contiguous()),
           "walk_ms_plain": time_walk(ht, s, "plain")}
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
