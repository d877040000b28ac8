"""Host side of the lightcone / halo-record stage, on the CPU: the cosmology tables, the
oracle's restatement of the per-peak math, and the .pksc format, pinned on the reference's
own tests (test/test_cosmology.jl, test/test_catalog.jl)."""
import math

import numpy as np
import pytest

from oracle import catalog as oc


@pytest.fixture(scope="module")
def cosmo(ht):
    # the CosmologyParams of test_cosmology.jl
    return ht.catalog.CosmologyParams(Om=0.31, OB=0.049, OL=0.69, h=0.68, ns=0.965, s8=0.81)


@pytest.fixture(scope="module")
def chi2z6(ht, cosmo):
    return ht.catalog.build_chi_to_z(cosmo, z_max=6.0, npts=2000)


@pytest.fixture(scope="module")
def growth(ht, cosmo):
    return ht.catalog.dlinear_tables(cosmo)


def test_chi_to_z_round_trip(ht, cosmo, chi2z6):
    """test_cosmology.jl:72-91: chi(z) inverted through the 2000-point table within 0.005,
    0 below the table, z_max beyond it, and peak_redshift along an axis."""
    t = chi2z6
    for z in (0.0, 0.1, 0.5, 1.0, 2.0, 4.0, 5.9):
        c = ht.catalog.chi(z, cosmo)
        assert abs(oc.chi_to_z(t.chis, t.zs, t.z_max, c) - z) <= 0.005
    assert oc.chi_to_z(t.chis, t.zs, t.z_max, 0.0) == 0.0
    assert oc.chi_to_z(t.chis, t.zs, t.z_max, 1e10) == 6.0
    c1 = ht.catalog.chi(1.0, cosmo)
    assert abs(oc.peak_redshift((0, 0, 0), (c1, 0, 0), t.chis, t.zs, t.z_max) - 1.0) <= 0.005
    assert abs(oc.peak_redshift((100, 0, 0), (100 + c1, 0, 0), t.chis, t.zs, t.z_max) - 1.0) \
        <= 0.005


def test_growth_tables(ht, cosmo, growth):
    """Dlinear_tables is normalised to D(a=1) = 1 and lies inside test_cosmology.jl:26-27's
    bounds for the linear growth factor at z = 0.5 and 1 (0.75-0.82, 0.58-0.65)."""
    D = lambda z: oc.growth_D(growth, 1.0 / (1.0 + z))
    assert abs(D(0.0) - 1.0) < 1e-6
    assert 0.75 < D(0.5) < 0.82
    assert 0.58 < D(1.0) < 0.65
    assert D(2.0) < D(1.0) < D(0.5) < D(0.0)
    # outside the table: constant D/a times a
    assert oc.growth_D(growth, 10.0) == growth.D_a0 * 10.0
    assert oc.growth_D(growth, 1e-5) == growth.D_ainfty * 1e-5
    # within the table the 4-point interpolation reproduces the tabulated D/a at the nodes
    a = float(growth.atab[500])
    assert abs(oc.growth_D(growth, a) / a - growth.D_atab[500]) < 1e-12


def test_hunt_matches_bisect():
    xx = np.linspace(0.1, 2.0, 37)
    import bisect
    for x in (0.05, 0.1, 0.1000001, 0.9, 1.999, 2.0, 2.5):
        assert oc.hunt(xx, x) == bisect.bisect_left(list(xx), x)


def test_pksc_round_trip(ht, tmp_path):
    """test_catalog.jl:2-46: write/read keeps every field, the header and the empty case;
    33-field rows are recognised from the file size."""
    cat = ht.catalog
    rec = np.array([[1, 2, 3, .1, .2, .3, 5, .01, .02, .03, 100],
                    [10, 20, 30, 1, 2, 3, 8, .1, .2, .3, 200]], np.float32)
    p = tmp_path / "a.pksc"
    cat.write_pksc(str(p), rec, 8.0, 0.5)
    got, rmax, zo = cat.read_pksc(str(p))
    assert np.array_equal(got, rec) and rmax == np.float32(8.0) and zo == np.float32(0.5)
    raw = p.read_bytes()
    assert np.frombuffer(raw[:4], np.int32)[0] == 2 and len(raw) == 12 + 2 * 11 * 4
    cat.write_pksc(str(p), np.zeros((0, 11), np.float32), 0.0, 0.0)
    got, rmax, zo = cat.read_pksc(str(p))
    assert got.shape[0] == 0 and rmax == 0.0 and zo == 0.0
    ext = np.arange(3 * 33, dtype=np.float32).reshape(3, 33)
    cat.write_pksc(str(p), ext, 1.0, 2.0)
    got, _, _ = cat.read_pksc(str(p))
    assert got.shape == (3, 33) and np.array_equal(got, ext)


def test_oracle_records_match_host_packer(ht, growth):
    """Without a lightcone the oracle's basic records equal the host HaloRecord packer of
    the multi-rank path (dist.halo_records) given the same D and 2LPT coefficient."""
    rng = np.random.default_rng(3)
    npk, n, alatt, centre = 200, 64, 1.5, (10.0, -20.0, 30.0)
    i, j, k = (rng.integers(1, n + 1, npk).astype(np.int32) for _ in range(3))
    res = {"RTHL": np.where(rng.random(npk) < 0.6, rng.uniform(0.5, 5, npk), -1).astype(np.float32),
           "Fbarx": rng.normal(2, 1, npk).astype(np.float32),
           "Sbar": rng.normal(0, 3, 3 * npk).astype(np.float32),
           "Sbar2": rng.normal(0, 1, 3 * npk).astype(np.float32)}
    ZZon = 1.3
    rec = oc.halo_records({"i": i, "j": j, "k": k}, res, n, centre, alatt, growth, 0.31, 0.69,
                          ZZon=ZZon, ilpt=2)
    a = 1.0 / ZZon
    D = oc.growth_D(growth, a)
    coef = -3.0 / 7.0 * oc.omega_m_a(0.31, 0.69, a) ** (-1.0 / 143) * (D * D)
    pos = [[oc.cell_centre(c, alatt, int(v), n) for v in ax] for c, ax in zip(centre, (i, j, k))]
    host = ht.dist.halo_records(*pos, res, alatt, D=D, coef2=coef, ilpt=2)
    assert rec.shape == host.shape == (int((res["RTHL"] > 0).sum()), 11)
    assert np.array_equal(rec, host)
