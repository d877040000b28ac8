"""Pin the CPU oracle against the reference's own golden vectors and known answers.

Sources (guanyilun/Huntian.jl): test/test_radialshell_fortran.jl (Fortran get_homel
golden values), test/test_radialshell.jl (hRinteg, atab4, shells, eigen, synthetic
collapse / no-collapse), test/test_peakfind.jl (all cases), test/test_ellipsoidalcollapse.jl
and test/test_shell_gpu.jl (trilinear lookup).  No GPU needed.
"""
import hashlib
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN


def _cell(a, i, j, k, v):
    a[k - 1, j - 1, i - 1] = v


def fortran_peak_fields():
    """The 142^3 synthetic peak of test/test_radialshell_fortran.jl:26-51."""
    n = 142
    z = lambda: np.zeros((n, n, n), np.float32)
    d, ex, ey, ez = z(), z(), z(), z()
    _cell(d, 71, 71, 71, 10.0)
    for c in [(70, 71, 71), (72, 71, 71), (71, 70, 71), (71, 72, 71), (71, 71, 70), (71, 71, 72)]:
        _cell(d, *c, 5.0)
    for a, vals in ((ex, [.1, .05, .15, .1, .1, .1, .1]), (ey, [.2, .2, .2, .1, .3, .2, .2]),
                    (ez, [.3, .3, .3, .3, .3, .15, .45])):
        for c, v in zip([(71, 71, 71), (70, 71, 71), (72, 71, 71), (71, 70, 71), (71, 72, 71),
                         (71, 71, 70), (71, 71, 72)], vals):
            _cell(a, *c, v)
    return d, ex, ey, ez


FORTRAN = dict(fcrit=1.7161525487899780, RTHL=1.7320507764816284, Srb=1.9020472764968872,
               Fbarx=2.3230779170989990,
               Sbar=(2.5925926864147186E-02, 5.1851853728294373E-02, 7.7777773141860962E-02),
               strain_diag=(3.8717970252037048E-01, 7.7435940504074097E-01,
                            1.1615388393402100E+00),
               e_v=1.6666662693023682E-01, p_v=-5.1315236504478889E-08, zvir_half=-1.0)


def test_fixture_tables_intact():
    lines = open(os.path.join(GOLDEN, "tables.sha256")).read().split("\n")
    for ln in filter(None, lines):
        digest, name = ln.split()
        assert hashlib.sha256(open(os.path.join(GOLDEN, name), "rb").read()).hexdigest() == digest


@pytest.mark.parametrize("kind", ["radialshell", "shellgpu", "cudakernel"])
def test_fortran_golden(oracle, fortran_table_path, kind):
    d, ex, ey, ez = fortran_peak_fields()
    F = oracle.Fields(d, ex, ey, ez)
    ct = oracle.read_homeltab(fortran_table_path)
    shells = oracle.precompute_shells(8)
    ipp = 71 + 70 * 142 + 70 * 142 * 142
    r, code = oracle.analyse_peak(F, ipp, 1.0, 4, 1.0, 4.0, ct, shells,
                                  fcrit_override=FORTRAN["fcrit"], kind=kind)
    assert code == 0 and r["RTHL"] > 0
    # the reference test's tolerance is 1%; the restatement agrees to single precision
    rel = lambda a, b: abs(a - b) / abs(b)
    assert rel(r["RTHL"], FORTRAN["RTHL"]) < 1e-6
    assert rel(r["Srb"], FORTRAN["Srb"]) < 1e-6
    assert rel(r["Fbarx"], FORTRAN["Fbarx"]) < 1e-6
    for L in range(3):
        assert abs(r["Sbar"][L] - FORTRAN["Sbar"][L]) < 1e-7
        assert abs(r["Sbar2"][L]) < 1e-12
        assert abs(r["gradpk"][L]) < 1e-12 and abs(r["gradpkrf"][L]) < 1e-12
    S = r["strain"].reshape(3, 3, order="F")
    for L in range(3):
        assert rel(S[L, L], FORTRAN["strain_diag"][L]) < 1e-6
        for K in range(3):
            if K != L:
                assert abs(S[L, K]) < 1e-6
    assert rel(r["e_v"], FORTRAN["e_v"]) < 1e-6
    assert abs(r["p_v"] - FORTRAN["p_v"]) < 1e-7
    if kind == "shellgpu":
        assert r["zvir_half"] == 0.0      # analyse_peak_gpu does not compute it
    else:
        assert r["zvir_half"] == FORTRAN["zvir_half"]


def test_fcrit_from_table(oracle, fortran_table_path):
    ct = oracle.read_homeltab(fortran_table_path)
    # the Fortran run's fcrit came from the same table by a linear walk; the bisection
    # lands within the table's resolution of it
    assert abs(ct.fsc_of_z(0.0) - FORTRAN["fcrit"]) < 2e-3


def test_hRinteg_known_values(oracle):
    # test/test_radialshell.jl:3-30
    assert oracle.hRinteg(0.0, 0.0) == pytest.approx(-31.0 / 35.0, abs=1e-12)
    assert oracle.hRinteg(0.0, 1.5) == pytest.approx(1.4 * 1.5 - 31.0 / 35.0, abs=1e-12)
    assert oracle.hRinteg(2.0, 0.0) == 0.0
    assert oracle.hRinteg(3.0, 1.0) == 0.0
    assert oracle.hRinteg(1.0, 0.0) == pytest.approx(-3.2 / 7.0, abs=1e-12)
    assert oracle.hRinteg(0.5, 2.0) == pytest.approx(oracle.hRinteg(-0.5, 2.0))
    assert oracle.hRinteg(0.5, 1.0) != oracle.hRinteg(0.5, 2.0)


def test_atab4(oracle):
    a = oracle.atab4()
    ca, cb = 3.0 / (2.0 * math.pi), 1.0 / (4.0 * math.pi)
    assert len(a) == 1101
    assert a[0] == pytest.approx(ca * 2.0 / 3.0, abs=1e-14)
    assert a[400] == 0.0 and a[499] == 0.0 and a[1099] == 0.0
    assert ca * (2.0 / 3.0 - 1.0 + 0.5) == pytest.approx(cb, abs=1e-14)


def test_precompute_shells(oracle):
    c1 = oracle.precompute_shells(1)
    assert len(c1) == 7 and c1[0, 3] == 0 and (c1[:, 3] <= 1).all()
    c2 = oracle.precompute_shells(2)
    assert len(c2) == 33 and (np.diff(c2[:, 3]) >= 0).all()
    # stable order inside a shell: dk outer, dj, di inner
    for r2 in np.unique(c2[:, 3]):
        rows = c2[c2[:, 3] == r2][:, :3]
        keys = [tuple(x) for x in rows[:, ::-1]]
        assert keys == sorted(keys)
    # shell counts of the hunt radii the configurations use (8, 24 and 35 cells)
    for rmax, ncells, nsh in [(8, 2109, 55), (24, 57777, 482), (35, 179579, 1024)]:
        c = oracle.precompute_shells(rmax)
        st, cnt, r2 = oracle.build_shell_tables(c)
        assert len(c) == ncells and len(r2) == nsh and cnt.sum() == ncells


def test_eigvals(oracle):
    assert np.allclose(oracle.eigvals_sym3(np.eye(3)), [1, 1, 1], atol=1e-12)
    assert np.allclose(oracle.eigvals_sym3(np.diag([1.0, 2.0, 3.0])), [1, 2, 3], atol=1e-12)
    rng = np.random.default_rng(3)
    for _ in range(200):
        a = rng.standard_normal((3, 3)) * rng.uniform(1e-3, 1e3)
        s = (a + a.T) / 2
        ref = np.linalg.eigvalsh(s)
        assert np.allclose(oracle.eigvals_sym3(s), ref, rtol=1e-12,
                           atol=1e-13 * np.abs(ref).max())


def test_trilinear_exact_on_linear(oracle):
    # test/test_ellipsoidalcollapse.jl:115-137
    i, j, k = np.meshgrid(np.arange(11), np.arange(11), np.arange(11), indexing="ij")
    tab = (0.1 * i + 0.1 * j + 0.1 * k).astype(np.float32)   # (x, y, z) indexing
    ct = oracle.CollapseTable(tab.transpose(2, 1, 0), 0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    assert ct(0.0, 0.0, 0.0) == pytest.approx(0.0, abs=1e-5)
    assert ct(0.5, 0.0, 0.0) == pytest.approx(0.5, abs=1e-5)
    assert ct(0.0, 0.5, 0.0) == pytest.approx(0.5, abs=1e-5)
    assert ct(0.25, 0.25, 0.25) == pytest.approx(0.75, abs=1e-4)
    assert ct(-0.1, 0.0, 0.0) == -1.0
    assert ct(1.1, 0.0, 0.0) == -1.0
    # test/test_shell_gpu.jl:422-450 query set, incl. corners and out-of-range
    for x, y, z in [(0, 0, 0), (.5, 0, .5), (1, 1, 0), (.25, .25, .25), (.37, .62, .13),
                    (.99, .01, .5)]:
        assert ct(x, y, z) == pytest.approx(x + y + z, abs=1e-5)
    assert ct(0.5, -0.2, 0.5) == -1.0


def _bump_grid(n, value, bump=None):
    d = np.full((n, n, n), value, np.float32)
    if bump is not None:
        c, v, w = bump
        for di in (-1, 0, 1):
            for dj in (-1, 0, 1):
                for dk in (-1, 0, 1):
                    _cell(d, c + di, c + dj, c + dk, w)
        _cell(d, c, c, c, v)
    z = np.zeros_like(d)
    return d, z, z.copy(), z.copy()


def test_synthetic_collapse_and_no_collapse(oracle):
    # test/test_radialshell.jl:85-139: zvir = 1 everywhere collapses, 100 everywhere not
    axes = (math.log10(1.5), math.log10(8.0), 0.0, 0.5, -1.0 + 1e-4, 1.0 - 1e-4)
    shells = oracle.precompute_shells(8)
    n = 20
    ipp = 10 + 9 * n + 9 * n * n
    F = oracle.Fields(*_bump_grid(n, 0.0, (10, 10.0, 5.0)))
    ct1 = oracle.CollapseTable(np.ones((3, 3, 5), np.float32), *axes)
    r, code = oracle.analyse_peak(F, ipp, 1.0, 4, 0.0, 4.0, ct1, shells)
    assert code == 0 and r["RTHL"] > 0 and r["Srb"] > 0
    F2 = oracle.Fields(*_bump_grid(n, 0.5))
    ct100 = oracle.CollapseTable(np.full((3, 3, 5), 100.0, np.float32), *axes)
    r2, code2 = oracle.analyse_peak(F2, ipp, 1.0, 4, 0.0, 4.0, ct100, shells)
    assert r2["RTHL"] == -1.0 and code2 != 0


# ---------------------------------------------------------- peak finding KATs ----
# test/test_peakfind.jl:4-115 (nbuff = 1, fcrit = 1)

def _pf(oracle, d, mask=None, max_peaks=2_000_000):
    mask = np.zeros(d.shape, np.int8) if mask is None else mask
    return oracle.find_peaks(d, mask, 1, 1.0, max_peaks), mask


def test_peakfind_kats(oracle):
    n = 11
    d = np.zeros((n, n, n), np.float32); _cell(d, 6, 6, 6, 2.0)
    (i, j, k, v), mask = _pf(oracle, d)
    assert list(zip(i, j, k)) == [(6, 6, 6)] and v[0] == 2.0 and mask[5, 5, 5] == 1
    assert len(_pf(oracle, np.full((n, n, n), 0.5, np.float32))[0][0]) == 0
    g = np.fromfunction(lambda k, j, i: (i + j + k + 3).astype(np.float32), (n, n, n))
    assert len(_pf(oracle, g.astype(np.float32))[0][0]) == 0
    m = np.zeros((n, n, n), np.int8); m[5, 5, 5] = 1
    assert len(_pf(oracle, d, m)[0][0]) == 0
    d2 = np.zeros((n, n, n), np.float32); _cell(d2, 1, 6, 6, 2.0)
    assert len(_pf(oracle, d2)[0][0]) == 0
    n = 15
    d3 = np.zeros((n, n, n), np.float32); _cell(d3, 4, 4, 4, 2.0); _cell(d3, 12, 12, 12, 3.0)
    (i, j, k, _), _ = _pf(oracle, d3)
    assert list(zip(i, j, k)) == [(4, 4, 4), (12, 12, 12)]
    d4 = np.zeros((n, n, n), np.float32)
    for c in [(4, 4, 4), (4, 4, 12), (12, 12, 4), (12, 12, 12)]:
        _cell(d4, *c, 2.0)
    (i, j, k, _), m4 = _pf(oracle, d4, max_peaks=2)
    # scan order k -> j -> i: (4,4,4) then (12,12,4)
    assert list(zip(i, j, k)) == [(4, 4, 4), (12, 12, 4)] and m4.sum() == 2


def test_peakfind_ties_accepted(oracle):
    n = 9
    d = np.zeros((n, n, n), np.float32)
    _cell(d, 4, 4, 4, 2.0); _cell(d, 5, 4, 4, 2.0)   # equal neighbours: both are peaks
    (i, j, k, _), _ = _pf(oracle, d)
    assert list(zip(i, j, k)) == [(4, 4, 4), (5, 4, 4)]


def test_oracle_conventions_agree_on_shared_outputs(oracle, julia_table_path):
    """analyse_peak and analyse_peak_gpu are the same criterion: on a smooth bump field
    they agree on every output except the documented convention differences."""
    rng = np.random.default_rng(7)
    n = 40
    z, y, x = np.meshgrid(*(np.arange(1, n + 1),) * 3, indexing="ij")
    d = np.zeros((n, n, n), np.float32)
    for c in [(20, 20, 20), (12, 27, 15)]:
        d += 3.0 * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / 18.0).astype(np.float32)
    d += 0.01 * rng.standard_normal(d.shape).astype(np.float32)
    eta = [(0.3 * rng.standard_normal(d.shape)).astype(np.float32) for _ in range(6)]
    lapd = (0.05 * rng.standard_normal(d.shape)).astype(np.float32)
    F = oracle.Fields(d, *eta, lapd=lapd)
    ct = oracle.read_homeltab(julia_table_path)
    shells = oracle.precompute_shells(10)
    for (ci, cj, ck) in [(20, 20, 20), (12, 27, 15)]:
        ipp = ci + (cj - 1) * n + (ck - 1) * n * n
        a, _ = oracle.analyse_peak(F, ipp, 1.0, 9, 1.0, 4.0, ct, shells, fcrit_override=1.0)
        b, _ = oracle.analyse_peak(F, ipp, 1.0, 9, 1.0, 4.0, ct, shells, fcrit_override=1.0,
                                   kind="cudakernel")
        assert a["RTHL"] > 0 and b["RTHL"] == a["RTHL"]
        for f in ("Fbarx", "e_v", "p_v", "Srb", "zvir_half"):
            assert b[f] == pytest.approx(a[f], rel=1e-12, abs=1e-15)
        for f in ("Sbar", "Sbar2", "gradpk", "gradpkf", "strain"):
            assert np.allclose(b[f], a[f], rtol=1e-12, atol=1e-15)
