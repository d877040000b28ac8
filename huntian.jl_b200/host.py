"""Host-side mirror of Huntian.jl's GPU halo-finder entry points.

`peak_find_tile_gpu` and `analyse_peaks_gpu_cuda_multirf` keep the names, argument
meaning and return values of the reference methods (ext/CUDAExt.jl:2938-3060 and
ext/CUDAExt.jl:2085-2344; stubs src/Huntian.jl:387-412 and :259-281) so a caller of the
reference finds the same entry points.  The compute runs in libhuntian_b200.so; torch is
used only for device memory, streams and the cuFFT smoothing that stays outside the path.

Layout: a field is a torch tensor (or numpy array) of shape (n3, n2, n1) in C order, i.e.
byte-for-byte Julia's column-major (n1, n2, n3) array; cell (i, j, k) (1-based) is
``a[k-1, j-1, i-1]``.  Index outputs are 1-based like the reference's.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import (HT_CONV_CPU, HT_CONV_GPU, HT_MODE_BATCHED, HT_MODE_LEARNED, HT_MODE_PLAIN,
                   RESULT_NAMES, RESULT_WIDTH, HtFields, HtPeakBatch, HtPeaks, HtResults,
                   check)

_CONV = {"gpu": HT_CONV_GPU, "cpu": HT_CONV_CPU}
_MODE = {"plain": HT_MODE_PLAIN, "batched": HT_MODE_BATCHED, "learned": HT_MODE_LEARNED}


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _stream_handle(stream: Optional[torch.cuda.Stream]) -> Optional[int]:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def _dev(x, dtype, device) -> Optional[torch.Tensor]:
    if x is None:
        return None
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(x), dtype=dtype, device=device)


def ir2min_of(Rf: float, alatt: float) -> int:
    """MultiResolution.jl:575-576: min(floor((1.75 Rf/alatt)^2), floor((40/alatt - 1)^2))."""
    return min(math.floor((1.75 * Rf / alatt) ** 2), math.floor((40.0 / alatt - 1) ** 2))


def nhunt_of(Rf_max: float, alatt: float, nbuff: int) -> int:
    """MultiResolution.jl:731-733: min(nbuff - 1, floor(1.75 Rf_max / alatt))."""
    return min(nbuff - 1, math.floor(Rf_max * 1.75 / alatt))


class HaloFinder:
    """A libhuntian_b200 context on one device: shell tables for hunt radius `nhunt`,
    the collapse table and the SPH table, reused across tiles and calls."""

    def __init__(self, nhunt: int, ct_table, X1, X2, Y1, Y2, Z1, Z2, *, out_val=-1.0,
                 device: int = 0):
        L = _lib.load()
        self.device = device
        self.nhunt = int(nhunt)
        tab = np.ascontiguousarray(np.asarray(ct_table, dtype=np.float32))
        if tab.ndim != 3:
            raise ValueError("collapse table must be 3-D, shape (nz, ny, nx)")
        nz, ny, nx = tab.shape
        self.axes = tuple(float(v) for v in (X1, X2, Y1, Y2, Z1, Z2))
        h = C.c_void_p()
        check(L.ht_ctx_create(device, self.nhunt, tab.ctypes.data, nx, ny, nz, *self.axes,
                              float(out_val), C.byref(h)))
        self._h = h
        ns, nc = C.c_int32(), C.c_int64()
        check(L.ht_ctx_shell_info(self._h, C.byref(ns), C.byref(nc)))
        self.nshells, self.ncells = ns.value, nc.value
        self._bound = None

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.load().ht_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def shell_r2(self) -> np.ndarray:
        out = np.zeros(self.nshells, np.int32)
        check(_lib.load().ht_ctx_shell_r2(self._h, out.ctypes.data, self.nshells))
        return out

    def fsc_of_z(self, z: float) -> float:
        v = C.c_double()
        check(_lib.load().ht_fsc_of_z(self._h, float(z), C.byref(v)))
        return v.value

    # ------------------------------------------------------------ smoothing ----
    def smooth_window(self, delta_k: torch.Tensor, n: int, boxsize: float, Rf: float,
                      wsmooth: int, out: Optional[torch.Tensor] = None, stream=None):
        """delta_k (complex64 rfft of an n^3 field, shape (n, n, n//2+1)) times the
        Float32 window of Filters.smooth_field (Filters.jl:72-99); out may alias delta_k."""
        if delta_k.dtype != torch.complex64 or tuple(delta_k.shape) != (n, n, n // 2 + 1):
            raise ValueError(f"delta_k must be complex64 of shape {(n, n, n // 2 + 1)}, got "
                             f"{delta_k.dtype} {tuple(delta_k.shape)}")
        delta_k = delta_k.contiguous()
        out = torch.empty_like(delta_k) if out is None else out
        check(_lib.load().ht_smooth_window(self._h, delta_k.data_ptr(), out.data_ptr(), int(n),
                                           float(boxsize), float(Rf), int(wsmooth),
                                           _stream_handle(stream)))
        return out

    def smooth_field(self, delta_k: torch.Tensor, n: int, boxsize: float, Rf: float,
                     wsmooth: int, work: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Filters.smooth_field: window (library kernel) then the cuFFT inverse rfft."""
        w = self.smooth_window(delta_k, n, boxsize, Rf, wsmooth, out=work)
        return torch.fft.irfftn(w, s=(n, n, n), dim=(0, 1, 2)).contiguous()

    def smooth_tile(self, delta_k: torch.Tensor, n: int, boxsize: float, Rf: float,
                    wsmooth: int, out: Optional[torch.Tensor] = None,
                    stream=None, planes: Optional[tuple] = None) -> torch.Tensor:
        """ht_smooth_tile: one filter of peak_find_tile_gpu (ext/CUDAExt.jl:2984-2989) --
        window (with the 1/n^3 folded in) + out-of-place cuFFT C2R of the tile's own rfft
        straight into an n^3 float32 tile."""
        if delta_k.dtype != torch.complex64 or tuple(delta_k.shape) != (n, n, n // 2 + 1):
            raise ValueError("delta_k must be the complex64 rfft of an n^3 tile")
        if not delta_k.is_contiguous():
            raise ValueError("delta_k must be contiguous (torch.fft.rfftn returns a strided "
                             "view on CUDA: call .contiguous() once per tile)")
        out = torch.empty((n, n, n), dtype=torch.float32, device=delta_k.device) \
            if out is None else out
        if planes is None:
            check(_lib.load().ht_smooth_tile(self._h, delta_k.data_ptr(), out.data_ptr(),
                                             int(n), float(boxsize), float(Rf), int(wsmooth),
                                             _stream_handle(stream)))
        else:   # only planes [lo, hi) are needed (the peak scan reads nbuff-1 .. n-nbuff)
            check(_lib.load().ht_smooth_tile_planes(self._h, delta_k.data_ptr(),
                                                    out.data_ptr(), int(n), float(boxsize),
                                                    float(Rf), int(wsmooth), int(planes[0]),
                                                    int(planes[1]), _stream_handle(stream)))
        return out

    @staticmethod
    def pencil_supported(n: int) -> bool:
        """Tile sides the pencil smoothing handles (576 and 1152)."""
        return bool(_lib.load().ht_smooth_pencil_supported(int(n)))

    def spectrum_pencil(self, delta_k: torch.Tensor, n: int, out: Optional[torch.Tensor] = None,
                        stream=None) -> torch.Tensor:
        """ht_spectrum_pencil: the tile's rfft (n, n, n//2+1) transposed once into pencils
        (n, n//2+1, n), kz contiguous, for ht_smooth_pencil."""
        if delta_k.dtype != torch.complex64 or tuple(delta_k.shape) != (n, n, n // 2 + 1):
            raise ValueError("delta_k must be the complex64 rfft of an n^3 tile")
        if not delta_k.is_contiguous():
            raise ValueError("delta_k must be contiguous")
        out = torch.empty((n, n // 2 + 1, n), dtype=torch.complex64, device=delta_k.device) \
            if out is None else out
        if out.data_ptr() == delta_k.data_ptr():
            raise ValueError("the pencil transpose is out of place")
        check(_lib.load().ht_spectrum_pencil(self._h, delta_k.data_ptr(), out.data_ptr(), int(n),
                                             _stream_handle(stream)))
        return out

    def smooth_pencil(self, pencil: torch.Tensor, n: int, boxsize: float, Rf: float,
                      wsmooth: int, lo: int, hi: int, out: Optional[torch.Tensor] = None,
                      stream=None) -> torch.Tensor:
        """ht_smooth_pencil: one filter of peak_find_tile_gpu from the pencil spectrum; only
        the rows out[z, y, :] with lo <= z, y < hi are written (the rows the peak scan of
        the inner region reads when lo = nbuff - 1, hi = n - nbuff + 1)."""
        if pencil.dtype != torch.complex64 or tuple(pencil.shape) != (n, n // 2 + 1, n) \
                or not pencil.is_contiguous():
            raise ValueError("pencil must be the contiguous output of spectrum_pencil")
        out = torch.empty((n, n, n), dtype=torch.float32, device=pencil.device) \
            if out is None else out
        check(_lib.load().ht_smooth_pencil(self._h, pencil.data_ptr(), out.data_ptr(), int(n),
                                           float(boxsize), float(Rf), int(wsmooth), int(lo),
                                           int(hi), _stream_handle(stream)))
        return out

    def smooth_box_wrapped(self, delta_k: torch.Tensor, n: int, nbuff: int, boxsize: float,
                           Rf: float, wsmooth: int, out: Optional[torch.Tensor] = None,
                           stream=None) -> torch.Tensor:
        """ht_smooth_filter: window + cuFFT inverse rfft of a periodic n^3 box, returned
        as the (n + 2 nbuff)^3 tile with periodic wrap (float32)."""
        if delta_k.dtype != torch.complex64 or tuple(delta_k.shape) != (n, n, n // 2 + 1):
            raise ValueError("delta_k must be the complex64 rfft of an n^3 box")
        nt = n + 2 * nbuff
        out = torch.empty((nt, nt, nt), dtype=torch.float32, device=delta_k.device) \
            if out is None else out
        check(_lib.load().ht_smooth_filter(self._h, delta_k.contiguous().data_ptr(),
                                           out.data_ptr(), int(n), int(nbuff), float(boxsize),
                                           float(Rf), int(wsmooth), _stream_handle(stream)))
        return out

    # ---------------------------------------------------------------- peaks ----
    def peakfind_filter(self, delta_s: torch.Tensor, mask: torch.Tensor, nbuff: int,
                        fcrit: float, filter_idx: int, max_peaks: int, out: dict,
                        lapd_s: Optional[torch.Tensor] = None, stream=None) -> None:
        n = delta_s.shape[-1]
        assert delta_s.is_contiguous() and delta_s.dtype == torch.float32
        assert mask.is_contiguous() and mask.dtype == torch.int8 and mask.shape == delta_s.shape
        pk = HtPeaks(out["i"].data_ptr(), out["j"].data_ptr(), out["k"].data_ptr(),
                     out["delta"].data_ptr(), _ptr(out.get("lapd")),
                     out["filter_idx"].data_ptr(), out["count"].data_ptr(),
                     _ptr(out.get("found")))
        check(_lib.load().ht_peakfind_filter(self._h, delta_s.data_ptr(), _ptr(lapd_s),
                                             mask.data_ptr(), n, int(nbuff), float(fcrit),
                                             int(filter_idx), int(max_peaks), C.byref(pk),
                                             _stream_handle(stream)))

    @staticmethod
    def alloc_peaks(max_peaks: int, device, with_lapd: bool) -> dict:
        z = lambda dt: torch.zeros(max(max_peaks, 1), dtype=dt, device=device)
        return {"i": z(torch.int32), "j": z(torch.int32), "k": z(torch.int32),
                "delta": z(torch.float32), "lapd": z(torch.float32) if with_lapd else None,
                "filter_idx": z(torch.int32),
                "count": torch.zeros(1, dtype=torch.int64, device=device),
                "found": torch.zeros(1, dtype=torch.int64, device=device)}

    # --------------------------------------------------------------- shells ----
    def bind_fields(self, delta, etax, etay, etaz, eta2x=None, eta2y=None, eta2z=None,
                    lapd=None, stream=None) -> None:
        """Bind a tile (device float32 tensors, cubic) and build its cell records."""
        ts = [delta, etax, etay, etaz, eta2x, eta2y, eta2z, lapd]
        for t in ts:
            if t is not None:
                assert t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()
                assert t.shape == delta.shape
        n3, n2, n1 = delta.shape
        f = HtFields(*[_ptr(t) for t in ts], n1, n2, n3)
        check(_lib.load().ht_fields_pack(self._h, C.byref(f), _stream_handle(stream)))
        self._bound = ts   # keep the caller's tensors alive while bound

    @staticmethod
    def alloc_results(npeaks: int, device, diagnostics: bool = False) -> dict:
        """The 14 result arrays; with diagnostics also the Int32 walk_shells and
        collapse_shell arrays."""
        out = {n: torch.empty(max(npeaks, 1) * RESULT_WIDTH.get(n, 1), dtype=torch.float32,
                              device=device) for n in RESULT_NAMES}
        if diagnostics:
            for n in _lib.DIAG_NAMES:
                out[n] = torch.empty(max(npeaks, 1), dtype=torch.int32, device=device)
        return out

    @staticmethod
    def _results_struct(out: dict) -> HtResults:
        return HtResults(*[out[n].data_ptr() for n in RESULT_NAMES],
                         *[_ptr(out.get(n)) for n in _lib.DIAG_NAMES])

    def analyse(self, pi, pj, pk, Rf, ir2min, ZZon, fcrit, alatt: float, *,
                rmax2rs: float = 0.0, nbuff: int = 0, mask: Optional[torch.Tensor] = None,
                conv: str = "gpu", mode: str = "batched", out: Optional[dict] = None,
                order: Optional[torch.Tensor] = None, cost: Optional[torch.Tensor] = None,
                stream=None) -> dict:
        """Shell collapse of the peaks (device tensors of equal length) on the bound tile.
        order: optional int32 processing order (a permutation of the peak indices); cost:
        float32 predicted walk cost per peak for mode="learned" (bracket.predict's high
        quantile).  Neither changes any result."""
        if self._bound is None:
            raise _lib.HTError(_lib.HT_ERR_STATE, "bind_fields() first")
        npk = int(pi.numel())
        if out is None:
            out = self.alloc_results(npk, pi.device)
        if order is not None:
            assert order.dtype == torch.int32 and order.numel() == npk and order.is_contiguous()
        if cost is not None:
            assert cost.dtype == torch.float32 and cost.numel() == npk and cost.is_contiguous()
        b = HtPeakBatch(pi.data_ptr(), pj.data_ptr(), pk.data_ptr(), Rf.data_ptr(),
                        ir2min.data_ptr(), ZZon.data_ptr(), fcrit.data_ptr(), npk, _ptr(order),
                        _ptr(cost))
        r = self._results_struct(out)
        check(_lib.load().ht_shell_analyse(self._h, C.byref(b), float(alatt), float(rmax2rs),
                                           int(nbuff), _ptr(mask), _CONV[conv], _MODE[mode],
                                           C.byref(r), _stream_handle(stream)))
        return out

    def analyse_static(self, fields: dict, pi, pj, pk, Rf, ir2min, ZZon, fcrit,
                       alatt: float, *, rmax2rs: float = 0.0, nbuff: int = 0,
                       mask: Optional[torch.Tensor] = None, conv: str = "gpu",
                       out: dict, stream=None) -> dict:
        """ht_shell_analyse_static: the same shell collapse with no device allocation in
        the call (for code under stream capture or with a caller-owned memory pool).
        `fields` maps delta, etax..etaz[, eta2x..eta2z, lapd] to device float32 tensors;
        `out` must be preallocated (alloc_results).  The library's 32 MiB static scratch
        is shared by all such calls: do not overlap them on the GPU."""
        g = lambda k: fields.get(k)
        n3, n2, n1 = fields["delta"].shape
        f = HtFields(*[_ptr(g(k)) for k in ("delta", "etax", "etay", "etaz", "eta2x", "eta2y",
                                             "eta2z", "lapd")], n1, n2, n3)
        b = HtPeakBatch(pi.data_ptr(), pj.data_ptr(), pk.data_ptr(), Rf.data_ptr(),
                        ir2min.data_ptr(), ZZon.data_ptr(), fcrit.data_ptr(), int(pi.numel()))
        r = HtResults(*[out[n].data_ptr() for n in RESULT_NAMES])
        check(_lib.load().ht_shell_analyse_static(self._h, C.byref(f), C.byref(b), float(alatt),
                                                  float(rmax2rs), int(nbuff), _ptr(mask),
                                                  _CONV[conv], C.byref(r),
                                                  _stream_handle(stream)))
        return out

    def record_gather_probe(self, idx: torch.Tensor, out: Optional[torch.Tensor] = None,
                            stream=None) -> torch.Tensor:
        """ht_record_gather_probe: the sum of each packed cell record at the 0-based cell
        indices `idx` (int64, device) of the bound tile, one 256-bit load each -- a
        measurement of scattered 32-byte gathers (NaN for an index outside the tile)."""
        assert idx.dtype == torch.int64 and idx.is_contiguous() and idx.is_cuda
        out = torch.empty(idx.numel(), dtype=torch.float32, device=idx.device) \
            if out is None else out
        check(_lib.load().ht_record_gather_probe(self._h, idx.data_ptr(), int(idx.numel()),
                                                 out.data_ptr(), _stream_handle(stream)))
        return out

    def last_stats(self):
        k, s, c = C.c_int64(), C.c_int64(), C.c_int64()
        check(_lib.load().ht_last_launch_stats(self._h, C.byref(k), C.byref(s), C.byref(c)))
        return {"kernels": k.value, "shells_walked": s.value, "cells_walked": c.value}

    def reject_counts(self) -> dict:
        """get_dump_counts (RadialShell.jl:28-32): why peaks ended without collapse, summed
        over every shell analysis on this finder since reset_reject_counts (synchronises
        the device).  Keys: premask, no_fcrit, m0_one, no_collapse, rthl_neg (the
        reference's counters) and outside (centres outside the bound tile)."""
        n = len(_lib.REJECT_REASONS)
        v = (C.c_int64 * n)()
        check(_lib.load().ht_reject_counts(self._h, v))
        return dict(zip(_lib.REJECT_REASONS, (int(x) for x in v)))

    def reset_reject_counts(self, stream=None) -> None:
        """reset_dump_counters! (RadialShell.jl:19-26), stream-ordered."""
        check(_lib.load().ht_reset_reject_counts(self._h, _stream_handle(stream)))

    def tune(self, block_bits: Optional[int] = None, pf_kz: Optional[int] = None,
             walk_bpsm: Optional[int] = None, fft_path: Optional[int] = None,
             wait_ns: Optional[int] = None, inject_tx: Optional[int] = None) -> None:
        """Set launch parameters (ht_ctx_tune); block_bits, pf_kz and walk_bpsm are
        result-neutral.  wait_ns is the limit of the bounded in-kernel waits; inject_tx is
        the test hook that makes the peak scan's first waits run out (0 = off)."""
        L = _lib.load()
        for key, v in ((_lib.HT_TUNE_BLOCK_BITS, block_bits), (_lib.HT_TUNE_PF_KZ, pf_kz),
                       (_lib.HT_TUNE_WALK_BPSM, walk_bpsm), (_lib.HT_TUNE_FFT_PATH, fft_path),
                       (_lib.HT_TUNE_WAIT_NS, wait_ns), (_lib.HT_TUNE_INJECT_TX, inject_tx)):
            if v is not None:
                check(L.ht_ctx_tune(self._h, key, int(v)))

    def device_status(self) -> int:
        """0 when every bounded in-kernel wait since the last call completed (synchronises
        the device and clears the word)."""
        v = C.c_int32()
        check(_lib.load().ht_device_status(self._h, C.byref(v)))
        return v.value


# ----------------------------------------------------------- reference mirrors ----

@dataclass
class ShellTables:
    """ShellAnalysisGPU.ShellTables (src/ShellAnalysisGPU.jl:28-36): the r^2-sorted cell
    offsets grouped into shells, 1-based shell_start like the reference's."""
    offsets_di: np.ndarray
    offsets_dj: np.ndarray
    offsets_dk: np.ndarray
    shell_start: np.ndarray
    shell_count: np.ndarray
    shell_r2: np.ndarray
    nshells: int

    @property
    def rmax(self) -> int:
        """The hunt radius the tables were built for (largest r with r^2 in the table)."""
        return math.isqrt(int(self.shell_r2[-1])) if self.nshells else 0


def build_shell_tables(rmax: int) -> ShellTables:
    """ShellAnalysisGPU.build_shell_tables (src/ShellAnalysisGPU.jl:44-71) over
    RadialShell.precompute_shells (src/HaloFinder/RadialShell.jl:151-166): every offset
    with r^2 <= rmax^2, generated dk-outer, dj, di-inner and stably sorted by r^2."""
    r = np.arange(-rmax, rmax + 1, dtype=np.int32)
    dk, dj, di = np.meshgrid(r, r, r, indexing="ij")   # di fastest, as the loops nest
    di, dj, dk = di.ravel(), dj.ravel(), dk.ravel()
    r2 = di * di + dj * dj + dk * dk
    keep = r2 <= rmax * rmax
    di, dj, dk, r2 = di[keep], dj[keep], dk[keep], r2[keep]
    o = np.argsort(r2, kind="stable")
    di, dj, dk, r2 = di[o], dj[o], dk[o], r2[o]
    edges = np.flatnonzero(np.diff(r2)) + 1
    start0 = np.concatenate([[0], edges]).astype(np.int64)
    count = np.diff(np.concatenate([start0, [len(r2)]])).astype(np.int64)
    return ShellTables(di.astype(np.int32), dj.astype(np.int32), dk.astype(np.int32),
                       start0 + 1, count, r2[start0].astype(np.int32), int(len(start0)))


@dataclass
class PeakCandidate:
    """PeakFind.PeakCandidate (PeakFind.jl:3-13), arrays over peaks."""
    i: np.ndarray
    j: np.ndarray
    k: np.ndarray
    ipp: np.ndarray
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    delta: np.ndarray
    Rsmooth: np.ndarray


def peak_find_tile_gpu(delta_tile, filters: Sequence, fcrits: Sequence[float], tile_masks_in,
                       xbx: float, ybx: float, zbx: float, alatt: float, nbuff: int,
                       wsmooth: int, ioutshear: int, *, threads: int = 256,
                       max_peaks: int = 2_000_000, finder: Optional[HaloFinder] = None,
                       device=None, return_device: bool = False):
    """Mirror of `peak_find_tile_gpu` (ext/CUDAExt.jl:2938-3060): rfft once, then per
    filter (in the given order, mask carried) smooth with cuFFT and run the library's
    peak scan.  `filters` are (id, fcrit, Rf) tuples as read_filterbank returns.
    Returns dict(peaks=PeakCandidate, Rf, FcRf, d2Rf, mask).  Unlike the reference the
    peak order is deterministic: filter order, then k/j/i scan order."""
    device = device or torch.device("cuda", torch.cuda.current_device())
    delta = _dev(delta_tile, torch.float32, device)
    n = delta.shape[-1]
    assert delta.shape == (n, n, n) and len(filters) == len(fcrits)
    if finder is None:
        raise ValueError("pass finder=HaloFinder(...) (the library context)")
    mask = _dev(tile_masks_in, torch.int8, device).clone()
    boxsize = n * float(alatt)   # periodic tile: boxsize_local = n * alatt
    has_lapd = ioutshear >= 1
    delta_k = torch.fft.rfftn(delta, dim=(0, 1, 2)).contiguous()
    pencil = None
    if HaloFinder.pencil_supported(n):   # transpose the spectrum once for every filter
        pencil = finder.spectrum_pencil(delta_k, n)
        del delta_k
    out = HaloFinder.alloc_peaks(max_peaks, device, has_lapd)
    ds = torch.empty((n, n, n), dtype=torch.float32, device=device)
    ls = torch.empty_like(ds) if has_lapd else None
    # the planes (and rows) the scan reads: nbuff - 1 .. n - nbuff
    lo, hi = max(0, int(nbuff) - 1), min(n, n - int(nbuff) + 1)
    for fi, (flt, fc) in enumerate(zip(filters, fcrits), start=1):
        Rf = float(flt[2])
        if pencil is not None:
            finder.smooth_pencil(pencil, n, boxsize, Rf, wsmooth, lo, hi, out=ds)
            if has_lapd:
                finder.smooth_pencil(pencil, n, boxsize, Rf, 3, lo, hi, out=ls)
        else:
            finder.smooth_tile(delta_k, n, boxsize, Rf, wsmooth, out=ds, planes=(lo, hi))
            if has_lapd:
                finder.smooth_tile(delta_k, n, boxsize, Rf, 3, out=ls, planes=(lo, hi))
        finder.peakfind_filter(ds, mask, nbuff, float(np.float32(fc)), fi, max_peaks, out,
                               lapd_s=ls)
    del ds, ls
    npk = int(out["count"].item())
    sl = lambda t: t[:npk]
    res_dev = {k: (sl(v) if v is not None and k not in ("count", "found") else v)
               for k, v in out.items()}
    if return_device:
        res_dev["mask"] = mask
        return res_dev
    i = sl(out["i"]).cpu().numpy().astype(np.int64)
    j = sl(out["j"]).cpu().numpy().astype(np.int64)
    k = sl(out["k"]).cpu().numpy().astype(np.int64)
    fidx = sl(out["filter_idx"]).cpu().numpy()
    fdelta = sl(out["delta"]).cpu().numpy()
    cen = 0.5 * (n + 1)
    Rfs = np.array([float(f[2]) for f in filters], dtype=np.float64)
    Rf_out = Rfs[fidx - 1] if npk else np.zeros(0)
    peaks = PeakCandidate(i, j, k, i + (j - 1) * n + (k - 1) * n * n,
                          xbx + alatt * (i - cen), ybx + alatt * (j - cen),
                          zbx + alatt * (k - cen), fdelta, Rf_out)
    d2 = sl(out["lapd"]).cpu().numpy() if has_lapd else np.zeros(npk, np.float32)
    return {"peaks": peaks, "Rf": Rf_out, "FcRf": fdelta, "d2Rf": d2,
            "mask": mask.cpu().numpy()}


def analyse_peaks_gpu_cuda_multirf(delta, etax, etay, etaz, eta2x, eta2y, eta2z, batches,
                                   stab, ct_table, X1, X2, Y1, Y2, Z1, Z2, alatt: float,
                                   ZZon: float, *, fcrit_override=None, ct=None,
                                   rmax2rs: float = 0.0, threads: int = 128,
                                   ct_out_val: float = -1.0, lapd=None, mask=None,
                                   nbuff: int = 0, finder: Optional[HaloFinder] = None,
                                   mode: str = "batched", conv: str = "gpu", device=None):
    """Mirror of `analyse_peaks_gpu_cuda_multirf` (ext/CUDAExt.jl:2085-2344).

    `batches` are (peaks_i, peaks_j, peaks_k, Rf, ir2min[, ZZon_pp, fcrit_pp]) tuples;
    `stab` is a ShellTables (build_shell_tables, the reference's type) or the hunt radius
    as an int.  All batches go to the library in ONE launch.  Returns (results, mask): a list with one dict of the 14
    output arrays per batch (host numpy, reference shapes (3, n) / (3, 3, n)), and the
    updated mask (numpy) or None.  Device-resident inputs are used in place."""
    device = device or torch.device("cuda", torch.cuda.current_device())
    if isinstance(stab, (int, np.integer)):
        nhunt = int(stab)
    elif isinstance(stab, ShellTables):
        nhunt = stab.rmax
    else:
        raise TypeError("stab must be a ShellTables (build_shell_tables) or an int hunt radius")
    if finder is None or finder.nhunt != nhunt:
        finder = HaloFinder(nhunt, ct_table, X1, X2, Y1, Y2, Z1, Z2, out_val=ct_out_val,
                            device=device.index or 0)
    if fcrit_override is not None:
        fcrit = float(fcrit_override)
    elif ct is not None:
        fcrit = ct.fsc_of_z(float(ZZon) - 1.0) if hasattr(ct, "fsc_of_z") else finder.fsc_of_z(float(ZZon) - 1.0)
    else:
        fcrit = 1.686
    f32 = lambda a: _dev(a, torch.float32, device)
    finder.bind_fields(f32(delta), f32(etax), f32(etay), f32(etaz),
                       f32(eta2x) if eta2x is not None else None,
                       f32(eta2y) if eta2y is not None else None,
                       f32(eta2z) if eta2z is not None else None,
                       f32(lapd) if lapd is not None else None)
    pis, pjs, pks, rfs, irs, zzs, fcs, sizes = [], [], [], [], [], [], [], []
    for b in batches:
        npk = len(b[0])
        sizes.append(npk)
        pis.append(np.asarray(b[0], np.int32)); pjs.append(np.asarray(b[1], np.int32))
        pks.append(np.asarray(b[2], np.int32))
        rfs.append(np.full(npk, float(b[3]))); irs.append(np.full(npk, int(b[4]), np.int32))
        if len(b) >= 7:
            zzs.append(np.asarray(b[5], np.float32)); fcs.append(np.asarray(b[6], np.float32))
        else:
            zzs.append(np.full(npk, np.float32(ZZon))); fcs.append(np.full(npk, np.float32(fcrit)))
    cat = lambda xs, dt: _dev(np.concatenate(xs) if xs else np.zeros(0), dt, device)
    pi, pj, pk = cat(pis, torch.int32), cat(pjs, torch.int32), cat(pks, torch.int32)
    Rf, ir2 = cat(rfs, torch.float64), cat(irs, torch.int32)
    zz, fc = cat(zzs, torch.float32), cat(fcs, torch.float32)
    mask_d = _dev(mask, torch.int8, device).clone() if mask is not None else None
    out = finder.analyse(pi, pj, pk, Rf, ir2, zz, fc, alatt, rmax2rs=rmax2rs, nbuff=nbuff,
                         mask=mask_d, conv=conv, mode=mode)
    host = {n: out[n].cpu().numpy() for n in RESULT_NAMES}
    results, off = [], 0
    for npk in sizes:
        r = {}
        for n in RESULT_NAMES:
            w = RESULT_WIDTH.get(n, 1)
            a = host[n][off * w:(off + npk) * w]
            r[n] = a.reshape(npk, 3, 3).transpose(2, 1, 0) if n == "strain" \
                else (a.reshape(npk, w).T if w > 1 else a)
        results.append(r)
        off += npk
    return results, (mask_d.cpu().numpy() if mask_d is not None else None)
