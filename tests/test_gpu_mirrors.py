"""The drop-in mirrors of the reference's two GPU entry points, called the way
run_multitile_split calls them (MultiResolution.jl:1036-1044 for peak_find_tile_gpu,
:532-644 for analyse_peaks_gpu_cuda_multirf), against the oracle.

peak_find_tile_gpu (ext/CUDAExt.jl:2938-3060): per filter the smoothed field (the same
library smoothing the mirror runs) goes through the oracle's find_peaks with the mask
carried; peak indices, PeakCandidate fields (ipp, x/y/z cell centres, delta, Rsmooth), Rf,
FcRf, d2Rf (ioutshear = 1: the Laplacian-filtered field at the peak) and the returned mask
must match exactly.  Both smoothing paths of the mirror are covered (a 64^3 tile through
ht_smooth_tile, a 576^3 tile through the pencil passes).

analyse_peaks_gpu_cuda_multirf (ext/CUDAExt.jl:2085-2344): several Rf batches in one call,
the 5-tuple form with the shared ZZon / fcrit and the 7-tuple form with per-peak ZZon and
fcrit (lightcone tiles), lapd given (d2F), mask in and out, fcrit from fcrit_override, from
a collapse table `ct` and from the 1.686 default; results per batch in the reference's
shapes ((n,), (3, n), (3, 3, n)) within the parity tolerance of oracle/parity.py, and the
returned mask equal to the oracle's.
"""
import numpy as np
import pytest
import torch

from gpu_helpers import to_dev

pytestmark = pytest.mark.gpu


def _bumps(n, rng, nb, noise=0.05, lo=6):
    z, y, x = np.meshgrid(*(np.arange(1, n + 1),) * 3, indexing="ij")
    d = noise * rng.standard_normal((n, n, n))
    for _ in range(nb):
        c = rng.integers(lo, n - lo + 1, 3)
        a, w = 1.0 + 2.5 * rng.random(), 6.0 + 20.0 * rng.random()
        d += a * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / w)
    return d.astype(np.float32)


def _mirror_vs_oracle(ht, oracle, d, nbuff, filters, fcrits, tab, axes, mask_cells):
    n = d.shape[0]
    alatt = 1.25
    xbx, ybx, zbx = 100.0, -40.0, 7.5
    mask_in = np.zeros((n, n, n), np.int8)
    for c in mask_cells:      # cells masked by earlier tiles / filters
        mask_in[c[2] - 1, c[1] - 1, c[0] - 1] = 1
    finder = ht.HaloFinder(4, tab, *axes)
    pf = ht.peak_find_tile_gpu(d, filters, fcrits, mask_in, xbx, ybx, zbx, alatt, nbuff, 1, 1,
                               finder=finder, max_peaks=1 << 20)
    # expected: the same library smoothing, the oracle's scan with the mask carried
    dk = torch.fft.rfftn(to_dev(d), dim=(0, 1, 2)).contiguous()
    pencil = ht.HaloFinder.pencil_supported(n)
    lo, hi = nbuff - 1, n - nbuff + 1
    pk = finder.spectrum_pencil(dk, n) if pencil else None
    mask = mask_in.copy()
    want = {c: [] for c in ("i", "j", "k", "delta", "Rf", "d2")}
    for fi, (flt, fc) in enumerate(zip(filters, fcrits), start=1):
        ds = torch.zeros((n, n, n), dtype=torch.float32, device="cuda")
        ls = torch.zeros_like(ds)
        if pencil:
            finder.smooth_pencil(pk, n, n * alatt, flt[2], 1, lo, hi, out=ds)
            finder.smooth_pencil(pk, n, n * alatt, flt[2], 3, lo, hi, out=ls)
        else:
            finder.smooth_tile(dk, n, n * alatt, flt[2], 1, out=ds, planes=(lo, hi))
            finder.smooth_tile(dk, n, n * alatt, flt[2], 3, out=ls, planes=(lo, hi))
        dsh, lsh = ds.cpu().numpy(), ls.cpu().numpy()
        i, j, k, dv = oracle.find_peaks(dsh, mask, nbuff, np.float32(fc))
        want["i"].append(i); want["j"].append(j); want["k"].append(k)
        want["delta"].append(dv); want["Rf"].append(np.full(len(i), float(flt[2])))
        want["d2"].append(lsh[k - 1, j - 1, i - 1])
    w = {c: np.concatenate(v) for c, v in want.items()}
    p = pf["peaks"]
    assert len(w["i"]) > 10
    assert np.array_equal(p.i, w["i"]) and np.array_equal(p.j, w["j"])
    assert np.array_equal(p.k, w["k"])
    assert np.array_equal(p.ipp, w["i"] + (w["j"] - 1) * n + (w["k"] - 1) * n * n)
    cen = 0.5 * (n + 1)
    assert np.array_equal(p.x, xbx + alatt * (w["i"] - cen))
    assert np.array_equal(p.y, ybx + alatt * (w["j"] - cen))
    assert np.array_equal(p.z, zbx + alatt * (w["k"] - cen))
    assert np.array_equal(p.delta, w["delta"]) and np.array_equal(pf["FcRf"], w["delta"])
    assert np.array_equal(p.Rsmooth, w["Rf"]) and np.array_equal(pf["Rf"], w["Rf"])
    assert np.array_equal(pf["d2Rf"], w["d2"])
    assert np.array_equal(pf["mask"], mask)
    # cells masked on entry never become peaks
    masked = {tuple(c) for c in mask_cells}
    assert not any((a, b, c) in masked for a, b, c in zip(p.i, p.j, p.k))
    finder.close()


def test_peak_find_tile_gpu_tile_path(ht, oracle, julia_table_path):
    rng = np.random.default_rng(11)
    tab, axes = ht.read_homeltab(julia_table_path)
    filters = [(1, 1.686, 6.0), (2, 1.686, 4.0), (3, 1.686, 2.5)]
    fcrits = [0.6, 0.45, 0.5]
    _mirror_vs_oracle(ht, oracle, _bumps(64, rng, 25), 8, filters, fcrits, tab, axes,
                      [(20, 20, 20), (33, 40, 29), (9, 50, 41)])


def test_peak_find_tile_gpu_pencil_path(ht, oracle, julia_table_path):
    # white noise (sigma 20): top-hat smoothed at 7.2 and 4 cells its rms is about 0.5 and
    # 1.2, so the thresholds keep the peaks above about 2 sigma
    g = torch.Generator().manual_seed(12)
    d = (20.0 * torch.randn((576,) * 3, generator=g)).numpy()
    tab, axes = ht.read_homeltab(julia_table_path)
    filters = [(1, 1.686, 9.0), (2, 1.686, 5.0)]
    fcrits = [1.0, 2.5]
    _mirror_vs_oracle(ht, oracle, d, 32, filters, fcrits, tab, axes,
                      [(100, 200, 300), (250, 250, 250)])


def _fields(n, rng):
    d = _bumps(n, rng, 14, lo=8)
    eta = [(0.3 * rng.standard_normal(d.shape)).astype(np.float32) for _ in range(3)]
    eta2 = [(0.15 * rng.standard_normal(d.shape)).astype(np.float32) for _ in range(3)]
    lapd = (0.05 * rng.standard_normal(d.shape)).astype(np.float32)
    return d, eta, eta2, lapd


def _oracle_batches(oracle, d, eta, eta2, lapd, batches, fc_shared, zz_shared, alatt, ct,
                    rmax, nbuff, mask):
    F = oracle.Fields(d, *eta, *eta2, mask=mask, lapd=lapd)
    out = []
    shells = oracle.precompute_shells(rmax)
    for b in batches:
        npk = len(b[0])
        zz = np.asarray(b[5], np.float64) if len(b) >= 7 else np.full(npk, zz_shared)
        fc = np.asarray(b[6], np.float64) if len(b) >= 7 else \
            np.full(npk, float(np.float32(fc_shared)))
        o, _ = oracle.analyse_batch(F, b[0], b[1], b[2], np.full(npk, b[4]), np.full(npk, b[3]),
                                    zz.astype(np.float32).astype(np.float64), fc, alatt, ct,
                                    shells, nbuff=nbuff, kind="cudakernel")
        out.append(o)
    return out


@pytest.mark.parametrize("fcrit_from", ["override", "ct", "default"])
def test_analyse_peaks_gpu_cuda_multirf(ht, oracle, julia_table_path, fcrit_from):
    from oracle import parity
    rng = np.random.default_rng(2025)
    n, nbuff, alatt, rmax = 56, 6, 1.0, 9
    d, eta, eta2, lapd = _fields(n, rng)
    i, j, k, _ = oracle.find_peaks(d, np.zeros(d.shape, np.int8), 1, 0.4)
    assert len(i) >= 12
    sel = rng.permutation(len(i))
    parts = np.array_split(sel, 3)
    zz_shared = 1.25
    tab, axes = ht.read_homeltab(julia_table_path)
    ct = oracle.read_homeltab(julia_table_path)
    batches = []
    for bi, (idx, Rf) in enumerate(zip(parts, (2.0, 3.5, 5.0))):
        b = (i[idx], j[idx], k[idx], Rf, ht.ir2min_of(Rf, alatt))
        if bi == 2:   # lightcone batch: per-peak ZZon and fcrit (the 7-tuple form)
            zz = (1.0 + 0.8 * rng.random(len(idx))).astype(np.float32)
            fc = np.array([np.float32(ct.fsc_of_z(float(z) - 1.0)) for z in zz], np.float32)
            b = b + (zz, fc)
        batches.append(b)
    kw = {}
    if fcrit_from == "override":
        kw["fcrit_override"] = 1.55
        fc_shared = 1.55
    elif fcrit_from == "ct":
        kw["ct"] = ct
        fc_shared = ct.fsc_of_z(zz_shared - 1.0)
    else:
        fc_shared = 1.686
    stab = ht.build_shell_tables(rmax)
    mask_in = np.zeros((n, n, n), np.int8)
    res, mask_out = ht.analyse_peaks_gpu_cuda_multirf(
        d, *eta, *eta2, batches, stab, tab, *axes, alatt, zz_shared, lapd=lapd,
        mask=mask_in, nbuff=nbuff, **kw)
    omask = mask_in.copy()
    want = _oracle_batches(oracle, d, eta, eta2, lapd, batches, fc_shared, zz_shared, alatt,
                           ct, rmax, nbuff, omask)
    assert len(res) == len(batches)
    total_collapsed = 0
    for r, o, b in zip(res, want, batches):
        npk = len(b[0])
        for name in ("RTHL", "Fbarx", "e_v", "p_v", "Srb", "d2F", "zvir_half"):
            assert r[name].shape == (npk,)
        for name in ("eigs", "Sbar", "Sbar2", "gradpk", "gradpkf", "gradpkrf"):
            assert r[name].shape == (3, npk)
        assert r["strain"].shape == (3, 3, npk)
        # back to per-peak rows in the oracle's layout (strain column-major per peak)
        g = {nm: (r[nm].T if r[nm].ndim == 2 else r[nm]) for nm in r}
        g["strain"] = np.stack([r["strain"][:, :, p].reshape(9, order="F")
                                for p in range(npk)]) if npk else np.zeros((0, 9))
        rep = parity.report(g, o)
        assert rep["flips_unexplained"] == 0, rep["flip_list"]
        assert rep["mismatches"] == 0, rep["mismatch_list"]
        total_collapsed += rep["collapsed"]
    assert total_collapsed > 0
    assert np.array_equal(mask_out, omask)
    # an int hunt radius is accepted in place of the tables
    res2, _ = ht.analyse_peaks_gpu_cuda_multirf(
        d, *eta, *eta2, batches, rmax, tab, *axes, alatt, zz_shared, lapd=lapd,
        nbuff=nbuff, **kw)
    for r, r2 in zip(res, res2):
        for name in r:
            assert np.array_equal(r[name], r2[name], equal_nan=True)


def test_multirf_rejects_unknown_stab(ht, julia_table_path):
    tab, axes = ht.read_homeltab(julia_table_path)
    z = np.zeros((8, 8, 8), np.float32)
    with pytest.raises(TypeError):
        ht.analyse_peaks_gpu_cuda_multirf(z, z, z, z, None, None, None, [], object(), tab,
                                          *axes, 1.0, 1.0)
