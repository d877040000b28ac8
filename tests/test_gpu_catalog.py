"""GPU parity of the lightcone state and halo-record packing (ht_peak_lightcone,
ht_pack_halos) with the oracle restatement of MultiResolution.jl:1097-1130 and
:1159-1219: redshifts, ZZon and kept peaks bit-exact, fcrit and the 2LPT-scaled fields
within one Float32 ulp (pow of the device vs the host), every other record field
bit-exact."""
import math

import numpy as np
import pytest
import torch

from oracle import catalog as oc
from gpu_helpers import to_dev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(ht, oracle, julia_table_path):
    cat = ht.catalog
    cosmo = cat.CosmologyParams()
    chi2z = cat.build_chi_to_z(cosmo, z_max=3.0, npts=2000)
    growth = cat.dlinear_tables(cosmo)
    tab, axes = ht.read_homeltab(julia_table_path)
    finder = ht.HaloFinder(6, tab, *axes)
    cat.set_cosmology(finder, cosmo, chi2z, growth)
    ct = oracle.read_homeltab(julia_table_path)
    return cat, cosmo, chi2z, growth, finder, ct


def _ulps(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    return np.abs(a - b)


def test_lightcone_matches_oracle(ht, setup):
    cat, cosmo, chi2z, growth, finder, ct = setup
    rng = np.random.default_rng(5)
    n, alatt, centre, npk = 128, 10.0, (2000.0, 100.0, -50.0), 4000
    i, j, k = (rng.integers(1, n + 1, npk).astype(np.int32) for _ in range(3))
    obs, z_max = (0.0, 0.0, 0.0), 0.8
    out = cat.peak_lightcone(finder, to_dev(i, torch.int32), to_dev(j, torch.int32),
                             to_dev(k, torch.int32), n, centre, alatt, obs, z_max)
    torch.cuda.synchronize()
    z, zz, fc, keep = oc.lightcone(i, j, k, n, centre, alatt, obs, chi2z.chis, chi2z.zs,
                                   chi2z.z_max, z_max, ct.fsc_of_z)
    assert np.array_equal(out["z"].cpu().numpy(), z)
    assert np.array_equal(out["ZZon"].cpu().numpy(), zz)
    assert _ulps(out["fcrit"].cpu().numpy(), fc).max() <= 1
    assert np.array_equal(out["keep"].cpu().numpy(), keep)
    assert 0 < len(keep) < npk


def test_lightcone_table_edges(ht, setup):
    """The observer inside the tile (z = 0 at its own cell) and peaks beyond the chi table
    (z clamps to the table's z_max, then the z <= z_max cut drops them)."""
    cat, cosmo, chi2z, growth, finder, ct = setup
    n, alatt = 16, 1000.0
    centre = (0.0, 0.0, 0.0)
    i = np.array([8, 9, 1, 16], np.int32)          # 8.5 is the tile centre
    j = np.array([8, 9, 1, 16], np.int32)
    k = np.array([8, 9, 1, 16], np.int32)
    obs = (-500.0, -500.0, -500.0)                 # the centre of cell (8, 8, 8)
    out = cat.peak_lightcone(finder, to_dev(i, torch.int32), to_dev(j, torch.int32),
                             to_dev(k, torch.int32), n, centre, alatt, obs, 2.5)
    torch.cuda.synchronize()
    z, zz, fc, keep = oc.lightcone(i, j, k, n, centre, alatt, obs, chi2z.chis, chi2z.zs,
                                   chi2z.z_max, 2.5, ct.fsc_of_z)
    g = out["z"].cpu().numpy()
    assert np.array_equal(g, z) and g[0] == 0.0 and g[3] == chi2z.z_max
    assert np.array_equal(out["keep"].cpu().numpy(), keep)


def _synthetic(rng, npk, n, with_d2=True):
    res = {"RTHL": np.where(rng.random(npk) < 0.6, rng.uniform(0.5, 6, npk), -1.0)
           .astype(np.float32)}
    res["RTHL"][7] = np.nan                       # packed by the reference (NaN <= 0 is false)
    for nm in ("Fbarx", "e_v", "p_v", "Srb", "d2F", "zvir_half"):
        res[nm] = rng.normal(0, 2, npk).astype(np.float32)
    for nm in ("Sbar", "Sbar2", "gradpk", "gradpkf", "gradpkrf", "eigs"):
        res[nm] = rng.normal(0, 3, 3 * npk).astype(np.float32)
    res["strain"] = rng.normal(0, 1, 9 * npk).astype(np.float32)
    peaks = {"i": rng.integers(1, n + 1, npk).astype(np.int32),
             "j": rng.integers(1, n + 1, npk).astype(np.int32),
             "k": rng.integers(1, n + 1, npk).astype(np.int32),
             "Rf": rng.uniform(1.5, 40, npk),
             "FcRf": rng.normal(2, 0.5, npk).astype(np.float32),
             "d2Rf": rng.normal(0, 1, npk).astype(np.float32) if with_d2 else None}
    return peaks, res


@pytest.mark.parametrize("ilpt,ioutshear,lightcone", [(2, 0, False), (1, 0, False),
                                                      (2, 1, True), (2, 0, True),
                                                      (1, 1, False)])
def test_pack_halos_matches_oracle(ht, setup, ilpt, ioutshear, lightcone):
    cat, cosmo, chi2z, growth, finder, ct = setup
    rng = np.random.default_rng(11 + ilpt + 2 * ioutshear)
    n, alatt, centre, npk = 96, 2.0, (300.0, -40.0, 12.5), 3000
    peaks, res = _synthetic(rng, npk, n, with_d2=ioutshear == 1 and lightcone)
    z_max = math.inf
    if lightcone:
        peaks["z"] = rng.uniform(0.0, 2.0, npk)
        z_max = 1.5
    dev_peaks = {"i": to_dev(peaks["i"], torch.int32), "j": to_dev(peaks["j"], torch.int32),
                 "k": to_dev(peaks["k"], torch.int32), "Rf": to_dev(peaks["Rf"], torch.float64),
                 "FcRf": to_dev(peaks["FcRf"]),
                 "d2Rf": to_dev(peaks["d2Rf"]) if peaks["d2Rf"] is not None else None,
                 "z": to_dev(peaks["z"], torch.float64) if lightcone else None}
    dev_res = {nm: to_dev(v) for nm, v in res.items()}
    got = cat.pack_halos(finder, dev_peaks, dev_res, n, centre, alatt, ZZon=1.25, z_max=z_max,
                         ilpt=ilpt, ioutshear=ioutshear).cpu().numpy()
    want = oc.halo_records(peaks, res, n, centre, alatt, growth, cosmo.Om, cosmo.OL,
                           ZZon=1.25, z_max=z_max, ilpt=ilpt, ioutshear=ioutshear)
    assert got.shape == want.shape and want.shape[0] > 1000
    exact = [c for c in range(got.shape[1]) if c not in (7, 8, 9)]
    assert np.array_equal(got[:, exact], want[:, exact], equal_nan=True)
    assert _ulps(got[:, 7:10], want[:, 7:10]).max() <= 1
    assert np.isnan(got[:, 6]).sum() == (0 if lightcone and peaks["z"][7] > z_max else 1)
    # a smaller cap writes the first rows only
    part = cat.pack_halos(finder, dev_peaks, dev_res, n, centre, alatt, ZZon=1.25,
                          z_max=z_max, ilpt=ilpt, ioutshear=ioutshear, cap=100).cpu().numpy()
    assert np.array_equal(part, got[:100], equal_nan=True)


def test_catalog_needs_tables(ht, julia_table_path):
    tab, axes = ht.read_homeltab(julia_table_path)
    f = ht.HaloFinder(6, tab, *axes)
    one = to_dev(np.ones(4, np.int32), torch.int32)
    with pytest.raises(ht.HTError) as e:
        ht.catalog.peak_lightcone(f, one, one, one, 8, (0, 0, 0), 1.0, (0, 0, 0), 1.0)
    assert "ht_ctx_set_cosmo" in str(e.value)


def test_tile_stage_with_lightcone(ht, setup):
    """The stage as the reference runs it on a lightcone: peak scan, per-peak redshift,
    ZZon and fcrit, the z cut, the collapse of the kept peaks with their own ZZon / fcrit,
    and the records of the collapsed ones (packed on the device, checked against the
    oracle's packing of the same collapse results)."""
    cat, cosmo, chi2z, growth, finder, ct = setup
    from gpu_helpers import gpu_find_peaks
    rng = np.random.default_rng(2)
    n, nbuff, alatt = 48, 6, 4.0
    delta = rng.normal(0, 1.2, (n, n, n)).astype(np.float32)
    etas = [rng.normal(0, 1, (n, n, n)).astype(np.float32) for _ in range(6)]
    peaks_np, _ = gpu_find_peaks(ht, finder, [delta], np.zeros((n, n, n), np.int8), nbuff, [1.2])
    i, j, k = (to_dev(peaks_np[c], torch.int32) for c in ("i", "j", "k"))
    centre, obs = (1500.0, 0.0, 0.0), (0.0, 0.0, 0.0)
    zs = cat.peak_lightcone(finder, i, j, k, n, centre, alatt, obs, 10.0)["z"]
    z_max = float(torch.quantile(zs, 0.5))          # keep about half of the peaks
    lc = cat.peak_lightcone(finder, i, j, k, n, centre, alatt, obs, z_max)
    keep = lc["keep"]
    assert 0 < keep.numel() < i.numel()
    d = {nm: to_dev(a) for nm, a in zip(("delta", "etax", "etay", "etaz", "eta2x", "eta2y",
                                          "eta2z"), [delta] + etas)}
    finder.bind_fields(d["delta"], d["etax"], d["etay"], d["etaz"], d["eta2x"], d["eta2y"],
                       d["eta2z"], None)
    m = keep.numel()
    Rf = torch.full((m,), 6.0, dtype=torch.float64, device="cuda")
    ir2 = torch.full((m,), ht.ir2min_of(6.0, alatt), dtype=torch.int32, device="cuda")
    sel = lambda t: t[keep].contiguous()
    res = finder.analyse(sel(i), sel(j), sel(k), Rf, ir2, sel(lc["ZZon"]), sel(lc["fcrit"]),
                         alatt, nbuff=nbuff)
    pk = {"i": sel(i), "j": sel(j), "k": sel(k), "Rf": Rf,
          "FcRf": sel(to_dev(peaks_np["delta"])), "d2Rf": None, "z": sel(lc["z"])}
    got = cat.pack_halos(finder, pk, res, n, centre, alatt, z_max=z_max, ioutshear=1)
    torch.cuda.synchronize()
    hres = {nm: v.cpu().numpy() for nm, v in res.items()}
    hpk = {nm: (v.cpu().numpy() if v is not None else None) for nm, v in pk.items()}
    want = oc.halo_records(hpk, hres, n, centre, alatt, growth, cosmo.Om, cosmo.OL,
                           z_max=z_max, ioutshear=1)
    got = got.cpu().numpy()
    assert got.shape == want.shape and got.shape[0] > 0
    exact = [c for c in range(33) if c not in (7, 8, 9)]
    assert np.array_equal(got[:, exact], want[:, exact], equal_nan=True)
    assert _ulps(got[:, 7:10], want[:, 7:10]).max() <= 1
