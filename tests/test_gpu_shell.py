"""Radial-shell collapse on the GPU vs the CPU FP64 oracle.

conv="gpu" is checked against the oracle's restatement of the reference CUDA kernels'
semantics (ShellAnalysisGPU.analyse_peak_gpu + zvir_half); conv="cpu" against
RadialShell.analyse_peak itself.  Tolerance: 1e-5 relative on every output (scaled by
the field's own magnitude with a small absolute floor), identical collapse decisions
and identical masks.  PLAIN and BATCHED modes must agree bit for bit.
"""
import numpy as np
import pytest

from gpu_helpers import compare, gpu_find_peaks, run_shell
from test_oracle_golden import FORTRAN, fortran_peak_fields

pytestmark = pytest.mark.gpu

REL = 1e-5
FLOOR = {"e_v": 1e-4, "p_v": 1e-4, "gradpk": 1e-4, "gradpkf": 1e-4, "gradpkrf": 1e-4,
         "Sbar": 1e-4, "Sbar2": 1e-4, "d2F": 1e-4, "strain": 1e-4, "eigs": 1e-4,
         "zvir_half": 1e-4}
KIND = {"gpu": "cudakernel", "cpu": "radialshell"}


def _fields(delta, eta, eta2=None, lapd=None):
    f = {"delta": delta, "etax": eta[0], "etay": eta[1], "etaz": eta[2], "lapd": lapd}
    if eta2 is not None:
        f.update(eta2x=eta2[0], eta2y=eta2[1], eta2z=eta2[2])
    return f


@pytest.mark.parametrize("conv", ["gpu", "cpu"])
@pytest.mark.parametrize("mode", ["plain", "batched"])
def test_fortran_golden_on_gpu(ht, fortran_table_path, conv, mode):
    d, ex, ey, ez = fortran_peak_fields()
    tab, axes = ht.read_homeltab(fortran_table_path)
    finder = ht.HaloFinder(8, tab, *axes)
    r, _ = run_shell(finder, _fields(d, (ex, ey, ez)), ([71], [71], [71]), 1.0, Rf=4.0,
                     ir2min=4, ZZon=1.0, fcrit=np.float32(FORTRAN["fcrit"]), conv=conv,
                     mode=mode)
    rel = lambda a, b: abs(a - b) / abs(b)
    assert rel(r["RTHL"][0], FORTRAN["RTHL"]) < 1e-6
    assert rel(r["Srb"][0], FORTRAN["Srb"]) < 1e-5
    assert rel(r["Fbarx"][0], FORTRAN["Fbarx"]) < 1e-5
    assert rel(r["e_v"][0], FORTRAN["e_v"]) < 1e-5
    assert abs(r["p_v"][0] - FORTRAN["p_v"]) < 1e-6
    S = r["strain"][0].reshape(3, 3, order="F")
    for L in range(3):
        assert rel(S[L, L], FORTRAN["strain_diag"][L]) < 1e-5
        assert abs(r["Sbar"][0][L] - FORTRAN["Sbar"][L]) < 1e-7
    assert r["zvir_half"][0] == -1.0


def _bump_field(n, centers, rng, noise=0.01, amp=3.0, width=18.0):
    z, y, x = np.meshgrid(*(np.arange(1, n + 1),) * 3, indexing="ij")
    d = np.zeros((n, n, n), np.float64)
    for c in centers:
        a, w = (amp, width) if len(c) == 3 else (c[3], c[4])
        d += a * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / w)
    d += noise * rng.standard_normal(d.shape)
    return d.astype(np.float32)


def _check(ht, oracle, finder, fields, peaks, alatt, Rf, ir2min, ZZon, fcrit, ct, rmax,
           conv, nbuff=0, allow_flips=0):
    n = fields["delta"].shape[0]
    mask0 = np.zeros((n, n, n), np.int8)
    g, gmask = run_shell(finder, fields, peaks, alatt, Rf=Rf, ir2min=ir2min, ZZon=ZZon,
                         fcrit=fcrit, nbuff=nbuff, mask=mask0, conv=conv)
    omask = mask0.copy()
    F = oracle.Fields(fields["delta"], fields["etax"], fields["etay"], fields["etaz"],
                      fields.get("eta2x"), fields.get("eta2y"), fields.get("eta2z"),
                      mask=omask, lapd=fields.get("lapd"))
    o, codes = oracle.analyse_batch(F, peaks[0], peaks[1], peaks[2], ir2min, Rf, ZZon,
                                    np.float32(fcrit), alatt, ct, oracle.precompute_shells(rmax),
                                    nbuff=nbuff, kind=KIND[conv])
    bad, flips = compare(g, o, REL, FLOOR)
    assert len(flips) <= allow_flips, f"collapse flips {flips}"
    assert not bad, f"{len(bad)} mismatching peaks, first: {bad[:5]}"
    if not flips:
        assert np.array_equal(gmask, omask)
    return g, o


@pytest.mark.parametrize("conv", ["gpu", "cpu"])
def test_bumps_flat_table(ht, oracle, conv):
    """test/test_shell_gpu.jl:567-676 construction: three Gaussian bumps, zvir = 0.5."""
    rng = np.random.default_rng(7777)
    n = 32
    d = _bump_field(n, [(16, 16, 16), (8, 8, 8), (24, 24, 24)], rng)
    eta = [(0.3 * rng.standard_normal(d.shape)).astype(np.float32) for _ in range(3)]
    eta2 = [(0.15 * rng.standard_normal(d.shape)).astype(np.float32) for _ in range(3)]
    lapd = (0.05 * rng.standard_normal(d.shape)).astype(np.float32)
    axes = (-2.0, 2.0, 0.0, 1.0, 0.0, 2.0)
    tab = np.full((10, 10, 10), 0.5, np.float32)
    finder = ht.HaloFinder(8, tab, *axes)
    ct = oracle.CollapseTable(tab, *axes)
    peaks = ([16, 8, 24], [16, 8, 24], [16, 8, 24])
    g, o = _check(ht, oracle, finder, _fields(d, eta, eta2, lapd), peaks, 1.0, 4.0, 4, 0.0,
                  1.0, ct, 8, conv)
    assert (g["RTHL"] > 0).all()


@pytest.mark.parametrize("conv", ["gpu", "cpu"])
def test_bumps_realistic_table_many_peaks(ht, oracle, julia_table_path, conv):
    """test/test_shell_gpu.jl:678-817 construction: 20 random bumps + noise, peaks from
    the peak finder, a real collapse table; both collapsing and non-collapsing peaks."""
    rng = np.random.default_rng(31415)
    n = 64
    centers = [(rng.integers(10, n - 9), rng.integers(10, n - 9), rng.integers(10, n - 9),
                1.0 + 2.0 * rng.random(), 15.0 + 10.0 * rng.random()) for _ in range(20)]
    d = _bump_field(n, centers, rng, noise=0.05)
    eta = [(0.3 * rng.standard_normal(d.shape)).astype(np.float32) for _ in range(3)]
    eta2 = [(0.15 * rng.standard_normal(d.shape)).astype(np.float32) for _ in range(3)]
    lapd = (0.05 * rng.standard_normal(d.shape)).astype(np.float32)
    i, j, k, _ = oracle.find_peaks(d, np.zeros(d.shape, np.int8), 1, 0.8)
    assert len(i) > 5
    tab, axes = ht.read_homeltab(julia_table_path)
    finder = ht.HaloFinder(10, tab, *axes)
    ct = oracle.read_homeltab(julia_table_path)
    g, o = _check(ht, oracle, finder, _fields(d, eta, eta2, lapd), (i, j, k), 1.0, 4.0, 4,
                  1.0, 1.0, ct, 10, conv)
    assert (g["RTHL"] > 0).sum() > 0 and (g["RTHL"] < 0).sum() > 0


def test_modes_bitwise_identical(ht, oracle, julia_table_path):
    rng = np.random.default_rng(5)
    n = 48
    centers = [(rng.integers(8, n - 7), rng.integers(8, n - 7), rng.integers(8, n - 7),
                1.5 + 2.0 * rng.random(), 10.0 + 20.0 * rng.random()) for _ in range(30)]
    d = _bump_field(n, centers, rng, noise=0.1)
    eta = [(0.3 * rng.standard_normal(d.shape)).astype(np.float32) for _ in range(6)]
    lapd = (0.05 * rng.standard_normal(d.shape)).astype(np.float32)
    i, j, k, _ = oracle.find_peaks(d, np.zeros(d.shape, np.int8), 2, 0.5)
    tab, axes = ht.read_homeltab(julia_table_path)
    finder = ht.HaloFinder(12, tab, *axes)
    f = _fields(d, eta[:3], eta[3:], lapd)
    outs = []
    for mode in ("plain", "batched"):
        r, m = run_shell(finder, f, (i, j, k), 1.5, Rf=3.0, ir2min=12, ZZon=1.0, fcrit=1.3,
                         nbuff=2, mask=np.zeros(d.shape, np.int8), mode=mode)
        outs.append((r, m))
    for key in outs[0][0]:
        assert np.array_equal(outs[0][0][key].view(np.int32), outs[1][0][key].view(np.int32)), key
    assert np.array_equal(outs[0][1], outs[1][1])


def test_processing_order_and_diagnostics(ht, oracle, julia_table_path):
    """Any processing order gives bit-identical results: PLAIN (batch order), BATCHED with
    the library's spatial order, BATCHED with a caller's random permutation.  The
    diagnostics agree across orders; collapse_shell brackets RTHL in radius."""
    rng = np.random.default_rng(77)
    n = 56
    centers = [(rng.integers(8, n - 7), rng.integers(8, n - 7), rng.integers(8, n - 7),
                1.5 + 2.0 * rng.random(), 10.0 + 20.0 * rng.random()) for _ in range(40)]
    d = _bump_field(n, centers, rng, noise=0.1)
    eta = [(0.3 * rng.standard_normal(d.shape)).astype(np.float32) for _ in range(6)]
    lapd = (0.05 * rng.standard_normal(d.shape)).astype(np.float32)
    i, j, k, _ = oracle.find_peaks(d, np.zeros(d.shape, np.int8), 2, 0.3)
    npk = len(i)
    assert npk > 40
    tab, axes = ht.read_homeltab(julia_table_path)
    finder = ht.HaloFinder(12, tab, *axes)
    f = _fields(d, eta[:3], eta[3:], lapd)
    # mixed filter radii so that both lane-group sizes occur
    Rf = np.where(np.arange(npk) % 3 == 0, 9.0, 2.5)
    ir2 = np.array([ht.ir2min_of(r, 1.2) for r in Rf], np.int32)
    runs = []
    for mode, order in (("plain", None), ("batched", None),
                        ("batched", rng.permutation(npk).astype(np.int32))):
        r, m = run_shell(finder, f, (i, j, k), 1.2, Rf=Rf, ir2min=ir2, ZZon=1.0, fcrit=1.3,
                         nbuff=2, mask=np.zeros(d.shape, np.int8), mode=mode, order=order,
                         diagnostics=True)
        runs.append((r, m))
    for r, m in runs[1:]:
        for key in runs[0][0]:
            assert np.array_equal(runs[0][0][key].view(np.int32), r[key].view(np.int32)), key
        assert np.array_equal(runs[0][1], m)
    r = runs[0][0]
    rad = np.sqrt(finder.shell_r2().astype(np.float64))   # rad[m - 1] of shell m
    col = r["RTHL"] > 0
    assert col.any() and (~col).any()
    assert np.all(r["collapse_shell"][~col] == 0)
    cs = r["collapse_shell"][col]
    assert np.all(cs >= 1)
    R = r["RTHL"][col].astype(np.float64)
    assert np.all(R >= rad[cs - 1] * (1 - 1e-6)) and np.all(R <= rad[cs] * (1 + 1e-6))
    assert np.all(r["walk_shells"][col] >= cs + 1)
    assert np.all(r["walk_shells"] >= 1)


def test_edge_peaks_near_tile_boundary(ht, oracle, julia_table_path):
    """Peaks whose shells leave the tile: out-of-tile cells are skipped, never wrapped."""
    rng = np.random.default_rng(11)
    n = 30
    centers = [(3, 4, 5, 3.0, 12.0), (27, 26, 2, 2.5, 20.0), (15, 2, 28, 2.0, 15.0)]
    d = _bump_field(n, centers, rng, noise=0.02)
    eta = [(0.2 * rng.standard_normal(d.shape)).astype(np.float32) for _ in range(3)]
    lapd = (0.05 * rng.standard_normal(d.shape)).astype(np.float32)
    tab, axes = ht.read_homeltab(julia_table_path)
    finder = ht.HaloFinder(9, tab, *axes)
    ct = oracle.read_homeltab(julia_table_path)
    peaks = ([3, 27, 15], [4, 26, 2], [5, 2, 28])
    for conv in ("gpu", "cpu"):
        _check(ht, oracle, finder, _fields(d, eta, None, lapd), peaks, 1.0, 3.0, 9, 1.0,
               1.0, ct, 9, conv, nbuff=3)


def test_large_filter_radius_gradient_window(ht, oracle, julia_table_path):
    """Rf/alatt far beyond the crossing radius: gradpkrf needs shells past the early
    exit point; the walk must still gather them (exactness vs the full walk)."""
    rng = np.random.default_rng(3)
    n = 40
    d = _bump_field(n, [(20, 20, 20, 4.0, 6.0)], rng, noise=0.05)
    eta = [(0.2 * rng.standard_normal(d.shape)).astype(np.float32) for _ in range(3)]
    tab, axes = ht.read_homeltab(julia_table_path)
    finder = ht.HaloFinder(16, tab, *axes)
    ct = oracle.read_homeltab(julia_table_path)
    peaks = ([20], [20], [20])
    for Rf in (1.0, 12.0, 15.0):
        _check(ht, oracle, finder, _fields(d, eta), peaks, 1.0, Rf, 4, 1.0, 1.0, ct, 16,
               "gpu")


def test_record_gather_probe(ht, julia_table_path):
    """ht_record_gather_probe reads the packed record of each given cell (delta, delta at the
    transposed cell, psi1 xyz, psi2 xyz) with the walk's 256-bit load: its sums equal the
    same FP32 sums of the fields; an index outside the tile gives NaN."""
    import torch
    from gpu_helpers import to_dev
    rng = np.random.default_rng(5)
    n = 24
    f = [rng.standard_normal((n, n, n)).astype(np.float32) for _ in range(7)]
    tab, axes = ht.read_homeltab(julia_table_path)
    finder = ht.HaloFinder(4, tab, *axes)
    finder.bind_fields(*[to_dev(a) for a in f])
    idx = rng.integers(0, n ** 3, 5000)
    idx[7] = n ** 3          # outside
    idx[11] = -1             # outside
    got = finder.record_gather_probe(torch.as_tensor(idx, dtype=torch.int64, device="cuda"))
    torch.cuda.synchronize()
    got = got.cpu().numpy()
    c = np.clip(idx, 0, n ** 3 - 1)
    i, j, k = c % n, (c // n) % n, c // (n * n)
    d = f[0]
    v = [d[k, j, i], d[j, i, k]] + [a[k, j, i] for a in f[1:]]   # delta[k, i, j] transposed
    want = ((v[0] + v[1]) + (v[2] + v[3])) + ((v[4] + v[5]) + (v[6] + v[7]))
    ok = (idx >= 0) & (idx < n ** 3)
    assert np.array_equal(got[ok], want[ok])
    assert np.isnan(got[~ok]).all()
    finder.close()
