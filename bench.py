"""Benchmark of the halo-finding hot path: peak finding + radial-shell collapse.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload tile1152|box512|box128|collapse_table] [--mode batched|plain]

Metric: candidate peaks per second carried through peak finding (all filters, mask
carried) and the radial-shell collapse, for one tile per GPU (weak scaling: N GPUs run N
independent tiles, no collective on the data path).  A step is one tile's halo-finding
stage as run_multitile_split performs it (MultiResolution.jl:1015-1219) with
peak_find_tile_gpu's smoothing (ext/CUDAExt.jl:2951-3012): one rfft of the tile, then per
filter the window + inverse FFT of the tile (the pencil passes at 576/1152, else
ht_smooth_tile) and the peak scan, then the cell-record pack, the shell collapse of every
peak in one launch, and the HaloRecord rows of the collapsed peaks (ht_pack_halos).

Inputs are seeded synthetic fields (BBKS LambdaCDM, Threefry noise, 2LPT), generated on
the device before timing; they are far larger than the 126 MB L2, so no flush is needed.
`--impl reference` times the CPU oracle (the C restatement of RadialShell.analyse_peak
and PeakFind.find_peaks) on the host cores on a bounded sample of the same workload.

`--workload collapse_table` measures the collapse-table generator instead (metric:
ellipsoids per second through the RK4 collapse, EllipsoidalCollapse.jl:492-590): a step
is the default 50 x 20 x 20 table (CollapseTable.jl:29-76) at the generator's default
cosmology, 20,000 independent ellipsoids, one per device thread.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

# tile1152 keeps ~150 GB resident (fields, cell records, spectrum, smoothing buffers): let
# the caching allocator grow segments instead of fragmenting across the per-step temporaries
os.environ.setdefault("PYTORCH_CUDA_ALLOC_CONF", "expandable_segments:True")
import torch  # noqa: E402

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (box cells per side, box size Mpc/h, nbuff, nfilters, Rmin, Rmax)
    "tile1152": dict(n=1024, L=1500.0, nbuff=64, nf=80, rmin=1.5, rmax=80.0,
                     desc="1024^3 core + 64-cell buffer = 1152^3 tile, L=1500 Mpc/h, "
                          "80 top-hat filters R=1.5-80 Mpc/h"),
    "box512": dict(n=512, L=1000.0, nbuff=54, nf=60, rmin=1.5, rmax=60.0,
                   desc="512^3 periodic box + 54-cell wrap = 620^3 tile, L=1000 Mpc/h, "
                        "60 top-hat filters R=1.5-60 Mpc/h"),
    "box128": dict(n=128, L=250.0, nbuff=36, nf=30, rmin=2.0, rmax=40.0,
                   desc="128^3 periodic box + 36-cell wrap = 200^3 tile, L=250 Mpc/h, "
                        "30 top-hat filters R=2-40 Mpc/h"),
    # the large tile's geometry at a size an ncu capture of the walk can replay
    "tile320": dict(n=192, L=281.25, nbuff=64, nf=80, rmin=1.5, rmax=80.0,
                    desc="192^3 core + 64-cell buffer = 320^3 tile at the 1152 tile's cell "
                         "size (L=281.25 Mpc/h, nhunt 63), 80 top-hat filters R=1.5-80 Mpc/h"),
}
METRIC = "peaks/s thru peakfind+shell collapse"
UNIT = "peaks/s"


def _package():
    name = "huntian_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg_dir = os.path.join(ROOT, "huntian.jl_b200")
    spec = importlib.util.spec_from_file_location(
        name, os.path.join(pkg_dir, "__init__.py"), submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def _peaks_json():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs"), "measured"
    return 6650.0, "fallback"


def _profile_traffic(workload):
    """DRAM bytes per walked cell of the walk kernel from the committed ncu summary
    (profiles/walk_traffic.txt); the caller scales it by the cells walked in this run."""
    p = os.path.join(ROOT, "profiles", "walk_traffic.txt")
    if not os.path.exists(p):
        return None
    vals = {}
    for ln in open(p):
        ln = ln.split("#")[0].split()
        if len(ln) == 2:
            vals[ln[0]] = float(ln[1])
    return vals.get(workload, vals.get("default"))


class Clocks:
    """nvidia-smi sampling during the timed region (start before, stop after)."""

    def __init__(self, index):
        try:
            import torch
            index = "GPU-" + str(torch.cuda.get_device_properties(index).uuid)
        except Exception:
            pass
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [ln.split(",") for ln in open(self.f.name).read().splitlines() if ln.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------- inputs ----

def make_inputs(ht, wl, seed, device):
    """Synthetic tile: delta, psi1, psi2 on the periodic box, wrapped to the tile (one tile
    with periodic cores, Parameters.jl:418-422)."""
    import torch
    from huntian_b200 import synth
    n, L, nbuff = wl["n"], wl["L"], wl["nbuff"]
    cosmo = synth.Cosmology()
    dk = synth.gaussian_box(n, L, seed, cosmo, device)
    psi1, psi2 = synth.displacements(dk, n, L, ilpt=2)
    tile = {"delta": synth.wrap_pad(synth._irfft(dk, n), nbuff)}
    del dk
    for nm, t in zip(("etax", "etay", "etaz"), psi1):
        tile[nm] = synth.wrap_pad(t, nbuff)
    for nm, t in zip(("eta2x", "eta2y", "eta2z"), psi2):
        tile[nm] = synth.wrap_pad(t, nbuff)
    del psi1, psi2
    torch.cuda.empty_cache()
    return tile


class Workload:
    def __init__(self, ht, name, seed, device, mode):
        self.ht, self.name, self.wl, self.mode = ht, name, WORKLOADS[name], mode
        wl = self.wl
        self.device = device
        self.n, self.nbuff = wl["n"], wl["nbuff"]
        self.nt = self.n + 2 * self.nbuff
        self.alatt = wl["L"] / self.n
        self.filters = ht.log_filterbank(wl["nf"], wl["rmin"], wl["rmax"])
        tab, axes = ht.read_homeltab(os.path.join(ROOT, "tests", "golden", "HomelTab_julia.dat"))
        self.nhunt = ht.nhunt_of(self.filters[0][2], self.alatt, self.nbuff)
        self.finder = ht.HaloFinder(self.nhunt, tab, *axes, device=device.index or 0)
        self.ZZon = 1.0                                   # z = 0
        self.fcrit = float(np.float32(self.finder.fsc_of_z(0.0)))
        self.tile = make_inputs(ht, wl, seed, device)
        self.boxsize = self.nt * self.alatt           # the tile is FFT'd as periodic
        self.mask = torch.zeros((self.nt,) * 3, dtype=torch.int8, device=device)
        self.max_peaks = 48_000_000 if self.n >= 1024 else 6_000_000
        self.peaks = ht.HaloFinder.alloc_peaks(self.max_peaks, device, False)
        self.Rf_f = torch.tensor([f[2] for f in self.filters], dtype=torch.float64, device=device)
        self.ir2_f = torch.tensor([ht.ir2min_of(f[2], self.alatt) for f in self.filters],
                                  dtype=torch.int32, device=device)
        self.results = None
        self.npeaks = 0
        self.graph = None
        self.tuned = {}
        if mode == "learned":
            self.model = ht.bracket.BracketModel.load(device=device)
        self.pencil = ht.HaloFinder.pencil_supported(self.nt)
        # the stage ends with the halo records of the collapsed peaks (MultiResolution.jl:
        # 1159-1219): cosmology tables once, records packed on the device every step
        cat = ht.catalog
        cp = cat.CosmologyParams(Om=0.31, OB=0.049, OL=0.69, h=0.68, ns=0.965, s8=0.81)
        cat.set_cosmology(self.finder, cp, cat.build_chi_to_z(cp, z_max=3.0, npts=200),
                          cat.dlinear_tables(cp))
        self.halos = None

    def smooth(self, Rf):
        if getattr(self, "_ds", None) is None:
            self._ds = torch.empty((self.nt,) * 3, dtype=torch.float32, device=self.device)
        # only the planes (and, on the pencil path, the rows) the peak scan reads:
        # nbuff - 1 .. nt - nbuff
        lo, hi = self.nbuff - 1, self.nt - self.nbuff + 1
        if self.pencil:
            return self.finder.smooth_pencil(self.pk, self.nt, self.boxsize, Rf, 1, lo, hi,
                                             out=self._ds)
        return self.finder.smooth_tile(self.dk, self.nt, self.boxsize, Rf, 1, out=self._ds,
                                       planes=(lo, hi))

    def pf_loop(self, ev=None):
        """Per filter: window + inverse FFT of the tile (ht_smooth_pencil after one
        ht_spectrum_pencil transpose at 576/1152, else ht_smooth_tile), then the peak scan."""
        if self.pencil:
            if getattr(self, "pk", None) is None:
                self.pk = torch.empty((self.nt, self.nt // 2 + 1, self.nt),
                                      dtype=torch.complex64, device=self.device)
            self.finder.spectrum_pencil(self.dk, self.nt, out=self.pk)
        for fi, flt in enumerate(self.filters, start=1):
            ds = self.smooth(flt[2])
            if ev is not None:
                ev["pf"][fi - 1][0].record()
            self.finder.peakfind_filter(ds, self.mask, self.nbuff, self.fcrit, fi,
                                        self.max_peaks, self.peaks)
            if ev is not None:
                ev["pf"][fi - 1][1].record()

    def capture_graph(self):
        """Capture the per-filter loop (80 x [window table, window, cuFFT C2R, 4 peak-scan
        kernels] on tile1152) once into a CUDA graph, replayed every step."""
        self.dk = torch.empty((self.nt, self.nt, self.nt // 2 + 1), dtype=torch.complex64,
                              device=self.device)
        self.dk.copy_(torch.fft.rfftn(self.tile["delta"], dim=(0, 1, 2)))
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.pf_loop()          # sizes every workspace and cuFFT plan before capture
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.pf_loop()
        torch.cuda.synchronize()

    def step(self, ev=None, fields_ready=None, hooks=None):
        """One tile: peak scan over all filters, then pack + shell collapse.  fields_ready:
        an event after which the six displacement fields are on the device (they are first
        read by the pack, so their host copies may overlap the peak finding).  hooks: optional
        callables run on the host at the stage boundaries, where the end-to-end pipeline
        orders its copies: "start" (before the first write), "graph" (npk; the peaks are
        final), "pack" (delta and the displacement fields have been read), "walk" (before the
        walk writes the results and the mask), "end" (npk; results, mask, halos final)."""
        import torch
        call = lambda name, *a: hooks[name](*a) if hooks and name in hooks else None
        call("start")
        self.mask.zero_()
        self.peaks["count"].zero_()
        self.peaks["found"].zero_()
        graph = getattr(self, "graph", None)
        if graph is not None:
            # once per tile, into the buffer the graph reads
            self.dk.copy_(torch.fft.rfftn(self.tile["delta"], dim=(0, 1, 2)))
            if ev is not None:
                ev["pf"][0][0].record()
            graph.replay()
            if ev is not None:
                ev["pf"][0][1].record()
        else:
            self.dk = None
            # once per tile; torch returns a strided view, made contiguous once here
            self.dk = torch.fft.rfftn(self.tile["delta"], dim=(0, 1, 2)).contiguous()
            self.pf_loop(ev)
            self.dk = None
        npk = int(self.peaks["count"].item())
        self.npeaks = npk
        call("graph", npk)
        self.mask.zero_()                                # MultiResolution.jl:1083
        t = self.tile
        if ev is not None:
            ev["pack"][0].record()
        if fields_ready is not None:
            torch.cuda.current_stream().wait_event(fields_ready)
        self.finder.bind_fields(t["delta"], t["etax"], t["etay"], t["etaz"], t["eta2x"],
                                t["eta2y"], t["eta2z"], None)
        call("pack")
        if ev is not None:
            ev["pack"][1].record()
        fidx = self.peaks["filter_idx"][:npk].long() - 1
        Rf = self.Rf_f[fidx]
        ir2 = self.ir2_f[fidx]
        zz = torch.full((npk,), self.ZZon, dtype=torch.float32, device=self.device)
        fc = torch.full((npk,), self.fcrit, dtype=torch.float32, device=self.device)
        call("walk")
        if self.results is None or self.results["RTHL"].numel() < npk:
            self.results = self.ht.HaloFinder.alloc_results(npk, self.device)
        pi, pj, pk = self.peaks["i"][:npk], self.peaks["j"][:npk], self.peaks["k"][:npk]
        if ev is not None:
            ev["walk"][0].record()
        cost = None
        if self.mode == "learned":
            br = self.ht.bracket
            F = br.features(self.finder, pi, pj, pk, Rf, ir2, zz, fc, self.alatt,
                            peak_delta=self.peaks["delta"][:npk])
            cost = br.predict(self.finder, self.model, F)[:, 1].contiguous()
        self.finder.analyse(pi, pj, pk, Rf, ir2, zz, fc, self.alatt, nbuff=self.nbuff,
                            mask=self.mask, mode=self.mode, out=self.results, cost=cost)
        if ev is not None:
            ev["walk"][1].record()
        pks = {"i": pi, "j": pj, "k": pk, "Rf": Rf, "FcRf": self.peaks["delta"][:npk],
               "d2Rf": None, "z": None}
        if ev is not None and "records" in ev:
            ev["records"][0].record()
        self.halos = self.ht.catalog.pack_halos(self.finder, pks, self.results, self.nt,
                                                (0.0, 0.0, 0.0), self.alatt, ZZon=self.ZZon,
                                                ilpt=2, ioutshear=0)
        if ev is not None and "records" in ev:
            ev["records"][1].record()
        call("end", npk)
        return npk

    def _walk_args(self):
        npk = self.npeaks
        fidx = self.peaks["filter_idx"][:npk].long() - 1
        return (self.peaks["i"][:npk], self.peaks["j"][:npk], self.peaks["k"][:npk],
                self.Rf_f[fidx], self.ir2_f[fidx],
                torch.full((npk,), self.ZZon, dtype=torch.float32, device=self.device),
                torch.full((npk,), self.fcrit, dtype=torch.float32, device=self.device))

    def _cost(self, args):
        br = self.ht.bracket
        model = getattr(self, "model", None) or br.BracketModel.load(device=self.device)
        self.model = model
        F = br.features(self.finder, *args, self.alatt, peak_delta=self.peaks["delta"][:self.npeaks])
        return br.predict(self.finder, model, F)[:, 1].contiguous()

    def time_walk(self, reps=2, mode=None, out=None):
        """Walk-only timing on the current peaks (the autotuner's probe): the min over
        reps of CUDA events around the call (learned mode: with the features and the MLP)."""
        mode = mode or self.mode
        args = self._walk_args()
        best = None
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            self.mask.zero_()
            a.record()
            cost = self._cost(args) if mode == "learned" else None
            self.finder.analyse(*args, self.alatt, nbuff=self.nbuff, mask=self.mask,
                                mode=mode, out=out if out is not None else self.results,
                                cost=cost)
            b.record()
            torch.cuda.synchronize()
            t = a.elapsed_time(b)
            best = t if best is None else min(best, t)
        return best

    def walk_modes(self, reps=2):
        """The metric's comparison on this step's peaks: the walk (shell collapse of every
        peak, CUDA events) in the PLAIN mode (the reference's layout: fields read in place,
        peaks in batch order, static schedule), BATCHED (packed cell records, spatial
        order, persistent queue) and LEARNED (BATCHED ordered by the learned bracket, the
        features and the MLP inside the timed call), with a checksum of every result
        array and of the mask per mode: the three must be identical."""
        res = self.ht.HaloFinder.alloc_results(self.npeaks, self.device)
        out = {"walk_ms": {}, "checksum": {}}
        for mode in ("plain", "batched", "learned"):
            out["walk_ms"][mode] = self.time_walk(reps, mode, res)
            h = 0
            for k in self.ht.RESULT_NAMES:
                v = res[k][: self.npeaks * self.ht.RESULT_WIDTH.get(k, 1)].view(torch.int32)
                h = (h * 1000003 + int(v.long().sum().item())) % (1 << 61)
            h = (h * 1000003 + int(self.mask.long().sum().item())) % (1 << 61)
            out["checksum"][mode] = h
        ck = out["checksum"]
        out["identical"] = ck["plain"] == ck["batched"] == ck["learned"]
        w = out["walk_ms"]
        out["speedup_learned_vs_plain"] = w["plain"] / w["learned"]
        out["speedup_learned_vs_batched"] = w["batched"] / w["learned"]
        return out

    def gather_ceiling(self, n=1 << 26, reps=5):
        """The rate of scattered 32-byte record gathers with no reuse: uniformly random cells
        of the packed tile, one 256-bit load each (ht_record_gather_probe), CUDA events,
        mean of `reps` after a warm-up.  GB/s of gathered records."""
        ncell = self.nt ** 3
        g = torch.Generator(device=self.device).manual_seed(7)
        idx = torch.randint(0, ncell, (n,), device=self.device, generator=g, dtype=torch.int64)
        out = torch.empty(n, dtype=torch.float32, device=self.device)
        self.finder.record_gather_probe(idx, out)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            self.finder.record_gather_probe(idx, out)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / reps
        return {"gbs": n * 32 / ms / 1e6, "records": n, "ms": ms}

    def release_smoothing(self):
        """Drop the CUDA graph and the smoothing buffers (after the timed steps)."""
        self.graph = None
        self.pk = None
        self.dk = None
        self._ds = None
        torch.cuda.empty_cache()

    def autotune(self):
        """Pick the result-neutral launch parameters by timing them on this workload: the
        LEARNED block size (HT_TUNE_BLOCK_BITS) and the walk's blocks per SM."""
        chosen = {}
        if self.mode == "learned":
            t = {b: (self.finder.tune(block_bits=b), self.time_walk())[1] for b in (15, 16, 17, 18, 19)}
            chosen["block_bits"] = min(t, key=t.get)
            self.finder.tune(block_bits=chosen["block_bits"])
        t = {b: (self.finder.tune(walk_bpsm=b), self.time_walk())[1] for b in (2, 3)}
        chosen["walk_bpsm"] = min(t, key=t.get)
        self.finder.tune(walk_bpsm=chosen["walk_bpsm"])
        self.tuned = chosen
        return chosen


def run_ours(args, rank, world, device):
    import torch
    ht = _package()
    seed = args.seed + rank
    W = Workload(ht, args.workload, seed, device, args.mode)
    dist = world > 1
    W.step()
    torch.cuda.synchronize()
    if args.autotune:
        W.autotune()
    if args.graph:
        W.capture_graph()
    for _ in range(args.warmup - 1):
        W.step()
    torch.cuda.synchronize()
    stats = W.finder.last_stats()
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(device.index or 0) if rank == 0 else None
    W.finder.reset_reject_counts()          # stream-ordered, before the timed steps
    nf = len(W.filters)
    mk = lambda: torch.cuda.Event(enable_timing=True)
    evs = [{"pf": [(mk(), mk()) for _ in range(nf)], "pack": (mk(), mk()),
            "walk": (mk(), mk()), "records": (mk(), mk())} for _ in range(args.steps)]
    start, end = mk(), mk()
    start.record()
    tot_peaks = 0
    for s in range(args.steps):
        tot_peaks += W.step(evs[s])
    end.record()
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ck = clocks.stop() if clocks else None
    rejects = {k: v // args.steps for k, v in W.finder.reject_counts().items()}
    t_ms = start.elapsed_time(end)
    npf = nf if W.graph is None else 1    # with the graph one event pair spans the loop
    pf_ms = sum(a.elapsed_time(b) for e in evs for a, b in e["pf"][:npf]) / args.steps
    pack_ms = sum(e["pack"][0].elapsed_time(e["pack"][1]) for e in evs) / args.steps
    walk_ms = sum(e["walk"][0].elapsed_time(e["walk"][1]) for e in evs) / args.steps
    rec_ms = sum(e["records"][0].elapsed_time(e["records"][1]) for e in evs) / args.steps
    if dist:
        t = torch.tensor([t_ms, float(tot_peaks)], dtype=torch.float64, device=device)
        tmax = t.clone()
        torch.distributed.all_reduce(tmax[:1], op=torch.distributed.ReduceOp.MAX)
        torch.distributed.all_reduce(t[1:], op=torch.distributed.ReduceOp.SUM)
        t_ms, tot_peaks = float(tmax[0]), int(t[1])
    ms_per_step = t_ms / args.steps
    value = tot_peaks / (t_ms / 1e3)

    # e2e through the public mirror with host buffers: every rank runs its own tile's
    # pipeline; the whole job's rate is the peaks of all ranks over the slowest rank's time,
    # and the copied bytes are summed over the ranks
    if dist:
        torch.distributed.barrier()
    e2e = run_e2e(ht, W, args) if args.e2e_steps > 0 else None
    if dist and e2e is not None:
        e2e = ht.dist.aggregate_e2e(e2e)

    if rank != 0:
        return None
    peak_bw, peak_kind = _peaks_json()
    cells = stats["cells_walked"]
    alg_bytes = 32.0 * cells + 4.0 * 40 * W.npeaks   # 8 FP32 values per walked cell + outputs
    achieved = alg_bytes / (walk_ms / 1e3) / 1e9
    traffic = _profile_traffic(args.workload)
    if traffic is not None:
        traffic = float(traffic) * cells
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 fields, f64 sums + collapse",
        "data": "synthetic (seeded BBKS LambdaCDM Gaussian field, 2LPT)",
        "config": {"workload": args.workload, "desc": W.wl["desc"], "mode": args.mode,
                   "cuda_graph": bool(args.graph), "autotuned": W.tuned,
                   "peaks_per_step": W.npeaks, "halos_per_step": int(W.halos.shape[0]),
                   "nhunt": W.nhunt, "nshells": W.finder.nshells,
                   "fcrit": W.fcrit, "l2": "inputs (43 GB of fields) >> 126 MB L2, no flush",
                   "parallelism": f"tile-per-GPU x{world}"},
        "breakdown_ms": {"peakfind_kernels" if W.graph is None else
                         "smoothing_and_peakfind_graph": pf_ms, "pack": pack_ms,
                         "shell_walk": walk_ms, "halo_records": rec_ms,
                         "smoothing_fft_and_rest": ms_per_step - pf_ms - pack_ms - walk_ms -
                         rec_ms},
        "hot_path_peaks_per_s": W.npeaks / ((pf_ms + pack_ms + walk_ms) / 1e3),
        "roofline": {"kernel": "walk_kernel", "bound": "hbm", "achieved": achieved,
                     "peak": peak_bw, "unit": "GB/s", "frac": achieved / peak_bw,
                     "peak_source": peak_kind, "traffic": traffic,
                     "alg_bytes_per_launch": alg_bytes, "cells_walked": cells},
        # ours per step: per filter the window table (+ its kz rows on the pencil path),
        # 3 transform kernels (pencil passes, or the transposed path's window/transpose
        # kernels) and 4 peak-scan kernels; per step the pencil transpose, pack, order keys,
        # walk, halo flags and records (+ features and MLP in learned mode); cuFFT and CUB
        # launches not counted
        "gpu_launches": int(args.steps * ((9 if W.pencil else 8) * nf +
                                          (1 if W.pencil else 0) + 5 +
                                          (2 if args.mode == "learned" else 0))),
        "clocks": ck,
        "e2e": e2e,
    }
    # why the timed steps' peaks ended without collapse (the reference's counters,
    # RadialShell.jl:13-32, kept on the device), per step
    line["reject_counts_per_step"] = rejects
    line["post_step_ms"] = post_step(ht, W)
    line["walk_modes"] = W.walk_modes() if args.compare_modes else None
    # the walk's second ceiling: scattered 32-byte gathers with no reuse, measured here
    gc = W.gather_ceiling()
    line["roofline"]["random_gather_ceiling_gbs"] = gc["gbs"]
    line["roofline"]["frac_of_random_gather_ceiling"] = achieved / gc["gbs"]
    W.release_smoothing()
    if args.cpu_seconds > 0 and world == 1:   # the CPU leg and its parity: rank 0 at N = 1
        line["cpu_baseline"], line["parity"] = cpu_baseline(ht, W, args)
    return line


def post_step(ht, W, reps=3):
    """The stage after the step, outside the timed region: the Lagrangian exclusion of the
    step's halo records (Merger.merge_catalog, ht_merge_halos) without and with volume
    reduction, and the Eulerian positions of the survivors (finalize_eulerian), CUDA events
    on the current stream, mean of `reps` after one warm-up call."""
    import torch
    cat = ht.catalog
    rec = W.halos.contiguous()
    out = {"halos_in": int(rec.shape[0])}
    for name, kw in (("merge_halos", {}), ("merge_halos_volume_reduction",
                                          {"volume_reduction": True})):
        kept = cat.merge_halos(W.finder, rec, **kw)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            kept = cat.merge_halos(W.finder, rec, **kw)
        b.record()
        torch.cuda.synchronize()
        out[name] = a.elapsed_time(b) / reps
        out[name + "_kept"] = int(kept.shape[0])
    kept = cat.merge_halos(W.finder, rec)
    fin = kept.clone()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fin.copy_(kept)
        cat.finalize_eulerian(W.finder, fin, (0.0, 0.0, 0.0), ievol=0, z_out=0.0)
    b.record()
    torch.cuda.synchronize()
    out["finalize_eulerian"] = a.elapsed_time(b) / reps
    return out


def run_e2e(ht, W, args):
    """Same step through the public host-buffer API, K steps back to back: every step's
    fields start in pinned host memory and are copied into the device tile inside the timed
    region, and all of its results (peaks, the 14 result arrays, the mask and the halo
    records) are read back into pinned host buffers inside it.  The copies run on two copy
    streams beside the compute, ordered by events as a tile pipeline would: step s + 1's
    delta and displacement fields go up once step s's pack has read the tile (during step
    s's walk and step s + 1's peak finding; the pack of s + 1 waits for them), step s's
    peaks come down during its walk, and its results, mask (copied on the device into a
    read-back buffer first: the next step clears the mask the peak scan uses) and halo
    records during step s + 1's peak finding (the walk of s + 1 waits for them).  Only the
    first step's delta upload and the last step's read-back are not overlapped."""
    import torch
    host = {k: v.cpu().pin_memory() for k, v in W.tile.items()}
    h2d = sum(t.numel() * t.element_size() for t in host.values())
    names = [("peaks", c) for c in ("i", "j", "k", "delta", "filter_idx")] + \
        [("results", n) for n in ht.RESULT_NAMES]

    def out_count(grp, n, npk):
        return npk * (ht.RESULT_WIDTH.get(n, 1) if grp == "results" else 1)

    out_host = {n: torch.empty(out_count(g, n, W.npeaks), dtype=getattr(W, g)[n].dtype)
                .pin_memory() for g, n in names}
    out_host["mask"] = torch.empty(W.mask.shape, dtype=W.mask.dtype).pin_memory()
    out_host["halos"] = torch.empty(W.halos.numel(), dtype=torch.float32).pin_memory()
    mask_out = torch.empty_like(W.mask)
    main = torch.cuda.current_stream()
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    mk = lambda: torch.cuda.Event(enable_timing=True)
    K = max(1, args.e2e_steps)
    st = {"d2h": 0, "tot": 0, "peaks_done": None, "res_done": None}

    def upload():
        """delta, then the six displacement fields, on the upload stream."""
        with torch.cuda.stream(up):
            W.tile["delta"].copy_(host["delta"], non_blocking=True)
            d = torch.cuda.Event()
            d.record(up)
            for k, v in host.items():
                if k != "delta":
                    W.tile[k].copy_(v, non_blocking=True)
            f = torch.cuda.Event()
            f.record(up)
        return d, f

    def fetch(dst, src):
        """Device -> pinned host copy on the download stream (src kept alive for it)."""
        if dst.numel() < src.numel():
            dst = torch.empty(src.numel(), dtype=src.dtype).pin_memory()
        with torch.cuda.stream(down):
            dst.reshape(-1)[:src.numel()].copy_(src.reshape(-1), non_blocking=True)
        src.record_stream(down)
        st["d2h"] += src.numel() * src.element_size()
        return dst

    def after(stream_wait):
        e = torch.cuda.Event()
        e.record(main)
        stream_wait.wait_event(e)

    ref_npk = W.npeaks                                  # the device-resident steps' count
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s0, s1 = mk(), mk()
    s0.record()
    up.wait_stream(main)
    ready = upload()
    for s in range(K):
        cur = {"ready": ready}
        st["d2h"] = 0

        def on_start(cur=cur):
            main.wait_event(cur["ready"][0])            # this step's delta is up
            if st["peaks_done"] is not None:            # the previous peaks are down
                main.wait_event(st["peaks_done"])

        def on_graph(npk):
            after(down)
            for grp, n in names[:5]:
                out_host[n] = fetch(out_host[n], W.peaks[n][:npk])
            e = torch.cuda.Event()
            e.record(down)
            st["peaks_done"] = e

        def next_inputs(s=s):
            if s + 1 < K:                               # the tile is free: next inputs up
                after(up)
                st["next"] = upload()

        def on_pack():
            if W.mode != "plain":                       # the walk reads the cell records
                next_inputs()

        def on_walk():
            if st["res_done"] is not None:              # the previous results are down
                main.wait_event(st["res_done"])

        def on_end(npk):
            if W.mode == "plain":                       # the walk read the fields in place
                next_inputs()
            mask_out.copy_(W.mask)                      # after the previous read-back (walk)
            after(down)
            for grp, n in names[5:]:
                out_host[n] = fetch(out_host[n], W.results[n][:out_count(grp, n, npk)])
            out_host["mask"] = fetch(out_host["mask"], mask_out)
            out_host["halos"] = fetch(out_host["halos"], W.halos)
            e = torch.cuda.Event()
            e.record(down)
            st["res_done"] = e

        npk = W.step(fields_ready=ready[1],
                     hooks={"start": on_start, "graph": on_graph, "pack": on_pack,
                            "walk": on_walk, "end": on_end})
        st["tot"] += npk
        ready = st.pop("next", None)
    main.wait_stream(down)
    main.wait_stream(up)
    s1.record()
    torch.cuda.synchronize()
    if st["tot"] != K * ref_npk:        # the same tile every step: the same peaks
        raise RuntimeError(f"end-to-end steps found {st['tot']} peaks, expected {K} x {ref_npk}")
    ms = s0.elapsed_time(s1)
    return {"value": st["tot"] / (ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(st["d2h"]), "ms_per_step": ms / K, "steps": K,
            "pipelined": "uploads of step s+1 and read-backs of step s overlap compute",
            "wall_s": time.perf_counter() - t0}


# ------------------------------------------------------------- CPU legs ----
#
# The reference's CPU path -- PeakFind.find_peaks over every filter with the mask carried,
# then RadialShell.analyse_peak per peak (src/HaloFinder/PeakFind.jl:15-78,
# src/HaloFinder/RadialShell.jl:281-865) -- timed on the host cores through the oracle (its
# C restatement, OpenMP over peaks as Pipeline.jl:235-242 threads them).  These legs call
# no function of the CUDA library: the fields come from synth (torch) and the smoothing
# from torch.fft with the top-hat window of Filters.smooth_field.  The walk of one peak
# of the large tile costs the CPU path about 0.1 s (every one of its 3,310 shells), so a
# step times a bounded sample: every filter's peaks in a central sub-volume (found by the
# oracle), a random sample of them analysed, and the find cost per cell of 130^3 blocks;
# the rate is per peak of that sample, extrapolated in no other way.

SUB = 64          # side of the central sub-volume whose peaks the CPU legs analyse
PARITY_PEAKS = 300


def torch_smooth(dk, n, boxsize, Rf):
    """Top-hat smoothed tile from its rfft (torch/cuFFT, not the library): the window
    3 (sin x - x cos x) / x^3 of Filters.smooth_field (ext/CUDAExt.jl:2853-2866) per integer
    |k|^2 in FP64, rounded to Float32, times the spectrum, inverse rfft."""
    import torch
    dev = dk.device
    q = np.arange(3 * (n // 2) ** 2 + 1, dtype=np.float64)
    x = np.sqrt(q) * (2 * math.pi / boxsize) * Rf
    with np.errstate(invalid="ignore", divide="ignore"):
        w = 3.0 * (np.sin(x) - x * np.cos(x)) / x ** 3
    w[0] = 1.0
    tab = torch.tensor(w.astype(np.float32), device=dev)
    iz = torch.arange(n, device=dev)
    sz = torch.where(iz <= n // 2, iz, iz - n)
    ix = torch.arange(n // 2 + 1, device=dev)
    out = torch.empty_like(dk)
    for z0 in range(0, n, 64):
        z1 = min(n, z0 + 64)
        qq = sz[z0:z1, None, None] ** 2 + sz[None, :, None] ** 2 + ix[None, None, :] ** 2
        out[z0:z1] = dk[z0:z1] * tab[qq]
    return torch.fft.irfftn(out, s=(n, n, n), dim=(0, 1, 2))


class CpuLeg:
    """The CPU path on a bounded sample of a tile workload (see the section comment)."""

    def __init__(self, tile, filters, alatt, nbuff, nhunt, fcrit, ZZon, table_path):
        import torch
        import oracle
        oracle.build()
        self.oracle = oracle
        self.nthreads = oracle.max_threads()
        self.filters, self.alatt, self.nbuff, self.nhunt = filters, alatt, nbuff, nhunt
        self.fcrit, self.ZZon = fcrit, ZZon
        self.ct = oracle.read_homeltab(table_path)
        self.shells = oracle.precompute_shells(nhunt)
        nt = tile["delta"].shape[0]
        self.nt = nt
        dk = torch.fft.rfftn(tile["delta"], dim=(0, 1, 2))
        # central sub-volume [s0, s0 + SUB) (0-based) on the tile's diagonal, so that the
        # transposed reads delta[k, i, j] of its walks stay inside the sub-tile below
        self.s0 = s0 = nt // 2 - SUB // 2
        self.o = o = s0 - nhunt - 1             # sub-tile origin (0-based)
        m = SUB + 2 * (nhunt + 1)
        self.sub = {k: np.ascontiguousarray(v[o:o + m, o:o + m, o:o + m].cpu().numpy())
                    for k, v in tile.items()}
        self.F = oracle.Fields(self.sub["delta"], self.sub["etax"], self.sub["etay"],
                               self.sub["etaz"], self.sub.get("eta2x"), self.sub.get("eta2y"),
                               self.sub.get("eta2z"))
        # every filter's peaks in the sub-volume (mask carried), and 130^3 blocks of some
        # filters' smoothed fields for the find timing
        mask = np.zeros((SUB + 2,) * 3, np.int8)
        pi, pj, pk, pf = [], [], [], []
        self.blocks = []
        c0, bsz = nbuff, 130
        step = max(1, len(filters) // 8)
        for fi, flt in enumerate(filters):
            ds = torch_smooth(dk, nt, nt * alatt, flt[2])
            blk = ds[s0 - 1:s0 + SUB + 1, s0 - 1:s0 + SUB + 1, s0 - 1:s0 + SUB + 1].cpu().numpy()
            i, j, k, _ = oracle.find_peaks(blk, mask, 1, fcrit)
            pi.append(i + s0 - 1); pj.append(j + s0 - 1); pk.append(k + s0 - 1)
            pf.append(np.full(len(i), fi))
            if fi % step == 0:
                self.blocks.append(np.ascontiguousarray(
                    ds[c0:c0 + bsz, c0:c0 + bsz, c0:c0 + bsz].cpu().numpy()))
            del ds
        del dk
        self.pi, self.pj, self.pk = (np.concatenate(v) for v in (pi, pj, pk))
        self.pf = np.concatenate(pf)
        self.Rf_all = np.array([f[2] for f in filters])
        self.ir2_all = np.array([min(math.floor((1.75 * f[2] / alatt) ** 2),
                                     math.floor((40.0 / alatt - 1) ** 2)) for f in filters])
        self.rng = np.random.default_rng(0)

    def analyse(self, pi, pj, pk, fidx, kind="radialshell", exact=False):
        """Oracle results for tile peaks (1-based tile coordinates) on the sub-tile."""
        o = self.o
        return self.oracle.analyse_batch(
            self.F, pi - o, pj - o, pk - o, self.ir2_all[fidx], self.Rf_all[fidx], self.ZZon,
            np.float32(self.fcrit), self.alatt, self.ct, self.shells, kind=kind,
            nthreads=self.nthreads, exact_products=exact)[0]

    def sample(self, budget):
        """One timed sample: find_peaks on the 130^3 blocks (one thread, as the
        reference's scan), analyse_peak on random sub-volume peaks (all threads)."""
        t_find, cells = 0.0, 0
        for blk in self.blocks:
            mask = np.zeros(blk.shape, np.int8)
            t0 = time.perf_counter()
            self.oracle.find_peaks(blk, mask, 1, self.fcrit)
            t_find += time.perf_counter() - t0
            cells += (blk.shape[0] - 2) ** 3
        per_cell = t_find / cells
        npk = len(self.pi)
        t_sh, done, batch = 0.0, 0, max(2 * self.nthreads, 32)
        while t_sh < budget and done < npk:
            idx = self.rng.choice(npk, size=min(batch, npk), replace=False)
            t0 = time.perf_counter()
            self.analyse(self.pi[idx], self.pj[idx], self.pk[idx], self.pf[idx])
            t_sh += time.perf_counter() - t0
            done += len(idx)
            batch = min(2 * batch, 2048)
        per_peak_shell = t_sh / max(done, 1)
        # find cost per peak: every filter scans every cell once; the sub-volume tells the
        # cells per peak of this workload
        per_peak_find = per_cell * len(self.filters) * SUB ** 3 / max(npk, 1)
        return {"value": 1.0 / (per_peak_shell + per_peak_find), "unit": UNIT,
                "cores": self.nthreads, "kind": "port",
                "sample": f"C restatement of RadialShell.analyse_peak (FP64, {self.nthreads} "
                          f"threads): {done} analyses of peaks drawn at random from the {npk} "
                          f"that find_peaks finds in the central {SUB}^3 sub-volume (all "
                          f"{len(self.filters)} "
                          f"filters, mask carried); find_peaks (1 thread) timed on 130^3 "
                          f"blocks of {len(self.blocks)} filters' fields; per-peak costs of "
                          f"this sample",
                "shell_s_per_peak": per_peak_shell, "find_s_per_cell": per_cell,
                "find_s_per_peak": per_peak_find}

    def parity(self, ht, finder, peaks, results, npk_all):
        """Device results of the timed step for step peaks inside the sub-volume (GPU
        convention, as the step ran) and the library's CPU convention on the same peaks,
        against both oracle variants (oracle/parity.py)."""
        import torch
        from oracle import parity
        s0 = self.s0
        pi, pj, pk = (peaks[c][:npk_all].cpu().numpy() for c in ("i", "j", "k"))
        inside = np.flatnonzero((pi - 1 >= s0) & (pi - 1 < s0 + SUB) & (pj - 1 >= s0) &
                                (pj - 1 < s0 + SUB) & (pk - 1 >= s0) & (pk - 1 < s0 + SUB))
        sel = np.sort(self.rng.choice(inside, size=min(PARITY_PEAKS, len(inside)),
                                      replace=False))
        fidx = peaks["filter_idx"][:npk_all].cpu().numpy()[sel] - 1
        width = ht.RESULT_WIDTH
        rows = lambda res, n, idx: {k: res[k][:n * width.get(k, 1)].cpu().numpy()
                                    .reshape(n, -1)[idx] for k in ("RTHL", "Fbarx", "e_v",
                                    "p_v", "Srb", "d2F", "zvir_half", "Sbar", "Sbar2", "gradpk",
                                    "gradpkf", "gradpkrf", "strain", "eigs")}
        out = {"peaks_in_subvolume": int(len(inside))}
        t0 = time.perf_counter()
        g_gpu = rows(results, npk_all, sel)
        ox = self.analyse(pi[sel], pj[sel], pk[sel], fidx, "cudakernel", exact=True)
        o = self.analyse(pi[sel], pj[sel], pk[sel], fidx, "cudakernel")
        out["gpu_convention"] = parity.report(g_gpu, o, ora_exact=ox, max_list=5)
        out["gpu_convention_vs_full_fp64"] = parity.report(g_gpu, ox, max_list=5)
        # the same peaks through the library's CPU convention (RadialShell.analyse_peak)
        dev = peaks["i"].device
        ti = lambda a: torch.as_tensor(a, dtype=torch.int32, device=dev)
        n = len(sel)
        res = finder.analyse(ti(pi[sel]), ti(pj[sel]), ti(pk[sel]),
                             torch.as_tensor(self.Rf_all[fidx], dtype=torch.float64, device=dev),
                             ti(self.ir2_all[fidx]),
                             torch.full((n,), self.ZZon, dtype=torch.float32, device=dev),
                             torch.full((n,), self.fcrit, dtype=torch.float32, device=dev),
                             self.alatt, conv="cpu", mode="plain")
        torch.cuda.synchronize()
        g_cpu = rows(res, n, np.arange(n))
        ox = self.analyse(pi[sel], pj[sel], pk[sel], fidx, "radialshell", exact=True)
        o = self.analyse(pi[sel], pj[sel], pk[sel], fidx, "radialshell")
        out["cpu_convention"] = parity.report(g_cpu, o, ora_exact=ox, max_list=5)
        out["oracle_s"] = time.perf_counter() - t0
        return out


def full_config1_cpu():
    """The reference's CPU path on the whole small box (128^3, L = 250 Mpc/h, 36-cell
    wrap, 30 top-hat filters R = 2-40 Mpc/h, seed 12345), unsampled: find_peaks over every
    filter (one thread, mask carried) and analyse_peak on every peak (all threads)."""
    import torch
    import oracle
    _package()
    from huntian_b200 import synth, tables
    n, L, nbuff, nf = 128, 250.0, 36, 30
    dev = torch.device("cuda", torch.cuda.current_device())
    cosmo = synth.Cosmology()
    dk0 = synth.gaussian_box(n, L, 12345, cosmo, dev)
    psi1, psi2 = synth.displacements(dk0, n, L, ilpt=2)
    tile = {"delta": synth.wrap_pad(synth._irfft(dk0, n), nbuff)}
    for nm, t in zip(("etax", "etay", "etaz", "eta2x", "eta2y", "eta2z"), psi1 + psi2):
        tile[nm] = synth.wrap_pad(t, nbuff)
    nt, alatt = n + 2 * nbuff, L / n
    filters = tables.log_filterbank(nf, 2.0, 40.0)
    ct = oracle.read_homeltab(os.path.join(ROOT, "tests", "golden", "HomelTab_julia.dat"))
    fcrit = float(np.float32(ct.fsc_of_z(0.0)))
    nhunt = min(nbuff - 1, math.floor(filters[0][2] * 1.75 / alatt))
    dk = torch.fft.rfftn(tile["delta"], dim=(0, 1, 2))
    host = {k: v.cpu().numpy() for k, v in tile.items()}
    mask = np.zeros((nt,) * 3, np.int8)
    t_find, found = 0.0, []
    for fi, flt in enumerate(filters):
        ds = torch_smooth(dk, nt, nt * alatt, flt[2]).cpu().numpy()
        t0 = time.perf_counter()
        i, j, k, _ = oracle.find_peaks(ds, mask, nbuff, fcrit)
        t_find += time.perf_counter() - t0
        found.append((i, j, k, np.full(len(i), fi)))
    pi, pj, pk, pf = (np.concatenate([f[c] for f in found]) for c in range(4))
    Rf = np.array([f[2] for f in filters])[pf]
    ir2 = np.array([min(math.floor((1.75 * f[2] / alatt) ** 2),
                        math.floor((40.0 / alatt - 1) ** 2)) for f in filters])[pf]
    F = oracle.Fields(host["delta"], host["etax"], host["etay"], host["etaz"], host["eta2x"],
                      host["eta2y"], host["eta2z"])
    nth = oracle.max_threads()
    t0 = time.perf_counter()
    o, _ = oracle.analyse_batch(F, pi, pj, pk, ir2, Rf, 1.0, np.float32(fcrit), alatt, ct,
                                oracle.precompute_shells(nhunt), nbuff=nbuff,
                                kind="radialshell", nthreads=nth)
    t_shell = time.perf_counter() - t0
    return {"value": len(pi) / (t_find + t_shell), "unit": UNIT, "cores": nth, "kind": "port",
            "sample": f"unsampled: the whole 128^3 box (200^3 tile, 30 filters): find_peaks "
                      f"over every filter ({t_find:.2f} s, 1 thread) and RadialShell."
                      f"analyse_peak on all {len(pi)} peaks ({t_shell:.1f} s, {nth} threads)",
            "peaks": int(len(pi)), "collapsed": int((o["RTHL"] > 0).sum()),
            "find_s": t_find, "shell_s": t_shell}


def cpu_baseline(ht, W, args):
    """Our arm's CPU leg (rank 0, N = 1, outside the timed region): the CPU path's rate on
    a bounded sample of this workload, and the parity of the timed step's results."""
    leg = CpuLeg(W.tile, W.filters, W.alatt, W.nbuff, W.nhunt, W.fcrit, W.ZZon,
                 os.path.join(ROOT, "tests", "golden", "HomelTab_julia.dat"))
    cb = leg.sample(args.cpu_seconds)
    par = leg.parity(ht, W.finder, W.peaks, W.results, W.npeaks)
    return cb, par


def run_reference(args, rank, world, device):
    """--impl reference: the reference's CPU path (the oracle) on the host cores, on
    bounded samples of the same workload; the CUDA library is never loaded."""
    if rank != 0:
        return None
    import torch
    _package()          # registers the package (synth, tables); the library stays unloaded
    from huntian_b200 import synth, tables
    wl = WORKLOADS[args.workload]
    n, L, nbuff = wl["n"], wl["L"], wl["nbuff"]
    alatt = L / n
    filters = tables.log_filterbank(wl["nf"], wl["rmin"], wl["rmax"])
    nhunt = min(nbuff - 1, math.floor(filters[0][2] * 1.75 / alatt))
    cosmo = synth.Cosmology()
    dk = synth.gaussian_box(n, L, args.seed, cosmo, device)
    psi1, psi2 = synth.displacements(dk, n, L, ilpt=2)
    tile = {"delta": synth.wrap_pad(synth._irfft(dk, n), nbuff)}
    del dk
    for nm, t in zip(("etax", "etay", "etaz", "eta2x", "eta2y", "eta2z"), psi1 + psi2):
        tile[nm] = synth.wrap_pad(t, nbuff)
    del psi1, psi2
    torch.cuda.empty_cache()
    import oracle
    tpath = os.path.join(ROOT, "tests", "golden", "HomelTab_julia.dat")
    fcrit = float(np.float32(oracle.read_homeltab(tpath).fsc_of_z(0.0)))
    leg = CpuLeg(tile, filters, alatt, nbuff, nhunt, fcrit, 1.0, tpath)
    del tile
    vals = [leg.sample(args.ref_seconds) for _ in range(args.warmup + args.steps)]
    vals = vals[args.warmup:]
    v = float(np.mean([c["value"] for c in vals]))
    cb = dict(vals[-1])
    cb["value"] = v
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * len(leg.pi) / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded BBKS LambdaCDM Gaussian field, 2LPT)",
            "config": {"workload": args.workload, "desc": wl["desc"],
                       "peaks_per_step": int(len(leg.pi)),
                       "step": f"the peaks of the central {SUB}^3 sub-volume"},
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.ref_full:
        line["cpu_baseline_full"] = full_config1_cpu()
    return line


def _collapse_metric(solver):
    name = "RK4" if solver == "rk4" else "Tsit5"
    return f"ellipsoids/s thru {name} collapse-table generation"


def _collapse_setup(ht, solver="rk4"):
    col, cat = ht.collapse, ht.catalog
    cp = cat.CosmologyParams(Om=0.315, OB=0.049, OL=0.685, h=0.674, ns=0.965, s8=0.808)
    ep = col.EllipsoidParams(cp, solver=solver)
    tp = col.CollapseTableParams()
    return cp, ep, tp


def _collapse_cpu(ep, tp):
    """The oracle's make_table (C restatement, OpenMP on every host thread), once."""
    from oracle import collapse as oc, max_threads
    eo = oc.EllipsoidOracle(ep.dlin_tables, ep.cosmo.Om, ep.cosmo.OL, solver=ep.solver)
    t0 = time.perf_counter()
    eo.make_table(tp.Nx, tp.Ny, tp.Nz, *tp.axes)
    dt = time.perf_counter() - t0
    n = tp.Nx * tp.Ny * tp.Nz
    return {"value": n / dt, "unit": "ellipsoids/s", "cores": max_threads(), "kind": "port",
            "sample": f"the whole {tp.Nx}x{tp.Ny}x{tp.Nz} table ({n} ellipsoids), or_make_table "
                      f"(C restatement of the {ep.solver} path, FP64, OpenMP)"}


def run_collapse_table(args, rank, world, device):
    """The collapse-table row: every rank builds the default table (replicas: the table
    is one small offline input).  value = ellipsoids per second of the device kernel over
    K launches (CUDA events on the launching stream, max over ranks); e2e = the host API
    ht_collapse_table (grid upload, launch, table download) timed around each call."""
    import torch
    ht = _package()
    cp, ep, tp = _collapse_setup(ht, args.solver)
    n = tp.Nx * tp.Ny * tp.Nz
    integ = ("RK4 tfac 0.01, nstepmax 10000" if args.solver == "rk4" else
             "Tsit5 abstol 1e-8 reltol 1e-6 (the reference's default :diffeq)")
    metric = _collapse_metric(args.solver)
    config = {"workload": "collapse_table", "solver": args.solver,
              "desc": f"{tp.Nx}x{tp.Ny}x{tp.Nz} zvir table (log10 Frho, e_v, p_v/e_v), "
                      f"{integ}, Planck 2018 (Om 0.315, OL 0.685)",
              "ellipsoids_per_step": n, "l2": "inputs 480 KB: compute bound, no flush",
              "parallelism": f"replicas x{world}"}
    if args.impl == "reference":
        if rank != 0:
            return None
        vals = [_collapse_cpu(ep, tp) for _ in range(args.warmup + args.steps)][args.warmup:]
        v = float(np.mean([c["value"] for c in vals]))
        cb = dict(vals[-1])
        cb["value"] = v
        return {"metric": metric, "value": v, "unit": "ellipsoids/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * n / v,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (the table's own grid)", "config": config,
                "impl": "reference", "cpu_baseline": cb,
                "e2e": {"value": v, "unit": "ellipsoids/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
    X1, X2, Y1, Y2, Z1, Z2 = tp.axes
    q = np.arange(n)
    i, j, k = q % tp.Nx, (q // tp.Nx) % tp.Ny, q // (tp.Nx * tp.Ny)
    x = X1 + i * ((X2 - X1) / (tp.Nx - 1))
    y = Y1 + j * ((Y2 - Y1) / (tp.Ny - 1))
    z = Z1 + k * ((Z2 - Z1) / (tp.Nz - 1))
    F = torch.tensor(np.power(10.0, x), dtype=torch.float64, device=device)
    E = torch.tensor(y, dtype=torch.float64, device=device)
    P = torch.tensor(z * y, dtype=torch.float64, device=device)
    for _ in range(args.warmup):
        ht.collapse.evolve_ellipses(F, E, P, ep, device=device.index or 0)
    torch.cuda.synchronize()
    clocks = Clocks(device.index or 0) if rank == 0 else None
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        ht.collapse.evolve_ellipses(F, E, P, ep, device=device.index or 0)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        t = torch.tensor([ms], device=device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    ck = clocks.stop() if clocks else None
    # end to end through the host API (grid upload, launch, table download)
    wall = []
    for _ in range(max(args.steps, 1)):
        t0 = time.perf_counter()
        ht.collapse.make_table(ep, tp, device=device.index or 0)
        wall.append(time.perf_counter() - t0)
    e2e_s = float(np.median(wall))
    ntab = len(ep.dlin_tables.atab)
    line = {"metric": metric, "value": world * n / (ms / 1e3), "unit": "ellipsoids/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (the table's own grid)", "config": config,
            "roofline": None,
            "roofline_note": "latency-bound FP64 chains (one ellipsoid per thread, ~10^3 "
                             "dependent RK4 steps); no HBM or tensor-core bound applies",
            "gpu_launches": args.steps, "clocks": ck,
            "e2e": {"value": world * n / e2e_s, "unit": "ellipsoids/s",
                    "h2d_bytes_per_step": 3 * n * 8 + 3 * ntab * 8,
                    "d2h_bytes_per_step": n * 8, "ms_per_step": 1e3 * e2e_s}}
    if rank == 0 and world == 1 and args.cpu_seconds > 0:
        line["cpu_baseline"] = _collapse_cpu(ep, tp)
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tile1152",
                    choices=list(WORKLOADS) + ["collapse_table"])
    ap.add_argument("--mode", default="learned", choices=["learned", "batched", "plain"])
    ap.add_argument("--solver", default="rk4", choices=["rk4", "diffeq"],
                    help="collapse_table workload: the integrator (the reference's two)")
    ap.add_argument("--graph", type=int, default=1,
                    help="capture the per-filter smoothing + peak-scan loop in a CUDA graph")
    ap.add_argument("--autotune", type=int, default=1,
                    help="time the result-neutral launch parameters once and keep the best")
    ap.add_argument("--seed", type=int, default=12345)
    ap.add_argument("--e2e-steps", type=int, default=8)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--ref-seconds", type=float, default=4.0,
                    help="CPU seconds of analyse_peak per step of --impl reference")
    ap.add_argument("--ref-full", type=int, default=1,
                    help="--impl reference also times the whole 128^3 box unsampled")
    ap.add_argument("--compare-modes", type=int, default=1,
                    help="after the timed steps, time the walk in the PLAIN, BATCHED and "
                         "LEARNED modes on the same peaks")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                             device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if args.workload == "collapse_table":
        line = run_collapse_table(args, rank, world, device)
    elif args.impl == "reference":
        line = run_reference(args, rank, world, device)
    else:
        line = run_ours(args, rank, world, device)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0 and line is not None:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
