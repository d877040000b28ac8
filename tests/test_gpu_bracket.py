"""Learned walk bracket on the GPU: the tensor-core inference and training kernels against
the CPU FP32 restatement (same BF16 rounding of every GEMM input), a training run that
reduces the loss, and the catalog under HT_MODE_LEARNED bit-identical to PLAIN whatever
the predicted costs."""
import os

import numpy as np
import pytest
import torch

from gpu_helpers import run_shell
from test_gpu_shell import _bump_field, _fields

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def finder(ht, julia_table_path):
    tab, axes = ht.read_homeltab(julia_table_path)
    return ht.HaloFinder(6, tab, *axes)


def _random_model(ht, seed):
    rng = np.random.default_rng(seed)
    br = ht.bracket
    p = br.init_params(seed)
    for b in ("b1", "b2", "b3", "b4"):
        o, s = br.OFFSETS[b]
        k = 2 if b == "b4" else s[0]
        p[o:o + k] = rng.normal(0, 0.2, k)
    mean = np.r_[rng.normal(0, 1, 12), np.zeros(4)].astype(np.float32)
    istd = np.r_[rng.uniform(0.5, 2, 12), np.zeros(4)].astype(np.float32)
    return p, mean, istd


def _features(rng, n):
    F = rng.normal(0, 1.5, (n, 16)).astype(np.float32)
    F[:, 12:] = 0
    return F


def test_inference_matches_cpu_reference(ht, finder):
    br = ht.bracket
    rng = np.random.default_rng(1)
    p, mean, istd = _random_model(ht, 1)
    model = br.BracketModel(p, mean, istd)
    for n in (1, 15, 16, 17, 1000):
        F = _features(rng, n)
        got = br.predict(finder, model, torch.as_tensor(F, device="cuda")).cpu().numpy()
        ref, _ = br.reference_forward(p, mean, istd, F)
        ref = ref.numpy()
        scale = np.abs(ref).max() + 1e-3
        # FP32 accumulation order differs (tensor-core vs CPU), which can move a hidden
        # activation across a BF16 rounding boundary: a few BF16 ulps of the output scale
        assert np.abs(got - ref).max() <= 3e-2 * scale, (n, np.abs(got - ref).max(), scale)
        assert np.median(np.abs(got - ref)) <= 2e-3 * scale
    # the tensor-core kernel reads the features with 16-byte loads: an unaligned view is
    # refused with a status, not read
    buf = torch.zeros(17 * 16 + 1, dtype=torch.float32, device="cuda")
    with pytest.raises(ht.HTError):
        br.predict(finder, model, buf[1:].view(17, 16))


def test_gradient_check_against_cpu(ht, finder):
    br = ht.bracket
    rng = np.random.default_rng(2)
    p, mean, istd = _random_model(ht, 2)
    model = br.BracketModel(p, mean, istd)
    n = 777
    F = _features(rng, n)
    ref_y, _ = br.reference_forward(p, mean, istd, F)
    t = (ref_y.numpy().mean(1) + rng.normal(0, 1.0, n)).astype(np.float32)
    g, loss = br.grad(finder, model, torch.as_tensor(F, device="cuda"),
                      torch.as_tensor(t, device="cuda"))
    g = g.cpu().numpy()
    ref = br.reference_grad(p, mean, istd, F, t)
    for name, (o, s) in br.OFFSETS.items():
        k = int(np.prod(s))
        a, b = g[o:o + k], ref[o:o + k]
        nb = np.linalg.norm(b)
        if nb == 0:
            assert np.abs(a).max() == 0, name
            continue
        assert np.linalg.norm(a - b) <= 2e-2 * nb, (name, np.linalg.norm(a - b) / nb)
    # padding rows / inputs stay untouched
    o, _ = br.OFFSETS["W4"]
    assert np.all(g[o + 128:o + 512] == 0)


def test_training_reduces_loss(ht, finder):
    br = ht.bracket
    rng = np.random.default_rng(3)
    n = 60000
    F = _features(rng, n)
    t = (5 + 2 * F[:, 0] - F[:, 3] * F[:, 4] + np.abs(F[:, 7]) +
         rng.normal(0, 0.3, n)).astype(np.float32)
    Fd, td = torch.as_tensor(F, device="cuda"), torch.as_tensor(t, device="cuda")
    m0 = br.BracketModel(br.init_params(0), F.mean(0), np.where(F.std(0) > 0, 1 / F.std(0), 0))
    _, l0 = br.grad(finder, m0, Fd, td)
    model = br.train(finder, Fd, td, epochs=8, batch=8192, lr=3e-3)
    _, l1 = br.grad(finder, model, Fd, td)
    assert float(l1) < 0.25 * float(l0), (float(l0), float(l1))
    pred = br.predict(finder, model, Fd).cpu().numpy()
    cover = np.mean((t >= pred[:, 0]) & (t <= pred[:, 1]))
    assert 0.6 < cover < 0.95, cover


def test_learned_mode_catalog_identical(ht, oracle, julia_table_path):
    rng = np.random.default_rng(21)
    n = 52
    centers = [(rng.integers(8, n - 7), rng.integers(8, n - 7), rng.integers(8, n - 7),
                1.5 + 2.0 * rng.random(), 10.0 + 20.0 * rng.random()) for _ in range(35)]
    d = _bump_field(n, centers, rng, noise=0.1)
    eta = [(0.3 * rng.standard_normal(d.shape)).astype(np.float32) for _ in range(6)]
    i, j, k, _ = oracle.find_peaks(d, np.zeros(d.shape, np.int8), 2, 0.3)
    npk = len(i)
    tab, axes = ht.read_homeltab(julia_table_path)
    finder = ht.HaloFinder(12, tab, *axes)
    f = _fields(d, eta[:3], eta[3:])
    Rf = np.where(np.arange(npk) % 3 == 0, 9.0, 2.5)
    ir2 = np.array([ht.ir2min_of(r, 1.2) for r in Rf], np.int32)
    base, bmask = run_shell(finder, f, (i, j, k), 1.2, Rf=Rf, ir2min=ir2, ZZon=1.0, fcrit=1.3,
                            nbuff=2, mask=np.zeros(d.shape, np.int8), mode="plain",
                            diagnostics=True)
    # learned mode with arbitrary costs (random, NaN, negative, huge) changes nothing
    cost = rng.normal(10, 20, npk).astype(np.float32)
    cost[::7] = np.nan
    cost[1::11] = 1e30
    dev = {kk: torch.as_tensor(v, device="cuda") if v is not None else None
           for kk, v in f.items()}
    finder.bind_fields(dev["delta"], dev["etax"], dev["etay"], dev["etaz"], dev["eta2x"],
                       dev["eta2y"], dev["eta2z"], None)
    b = lambda v, dt: torch.as_tensor(np.broadcast_to(np.asarray(v), (npk,)).copy(), dtype=dt,
                                      device="cuda")
    out = finder.alloc_results(npk, "cuda", diagnostics=True)
    for v in out.values():
        v.fill_(float("nan") if v.is_floating_point() else -7)
    mask = torch.zeros(d.shape, dtype=torch.int8, device="cuda")
    finder.analyse(b(i, torch.int32), b(j, torch.int32), b(k, torch.int32), b(Rf, torch.float64),
                   b(ir2, torch.int32), b(1.0, torch.float32), b(1.3, torch.float32), 1.2,
                   nbuff=2, mask=mask, mode="learned", out=out,
                   cost=torch.as_tensor(cost, device="cuda"))
    torch.cuda.synchronize()
    for key, v in base.items():
        g = out[key].cpu().numpy()[:v.size].reshape(v.shape)
        assert np.array_equal(g.view(np.int32), v.view(np.int32)), key
    assert np.array_equal(mask.cpu().numpy(), bmask)
    with pytest.raises(ht.HTError):
        finder.analyse(b(i, torch.int32), b(j, torch.int32), b(k, torch.int32),
                       b(Rf, torch.float64), b(ir2, torch.int32), b(1.0, torch.float32),
                       b(1.3, torch.float32), 1.2, nbuff=2, mode="learned", out=out)


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(
    os.path.abspath(__file__))), "huntian.jl_b200", "bracket_box512.npz")),
    reason="trained weights not present")
def test_shipped_weights_predict_walks(ht, oracle, julia_table_path):
    """The shipped model (trained on 512^3 synthetic tiles) loads and gives finite
    predictions for the peaks of a small bump field."""
    br = ht.bracket
    model = br.BracketModel.load()
    rng = np.random.default_rng(5)
    n = 48
    d = _bump_field(n, [(24, 24, 24, 3.0, 20.0), (12, 30, 20, 2.0, 10.0)], rng, noise=0.1)
    eta = [(0.3 * rng.standard_normal(d.shape)).astype(np.float32) for _ in range(3)]
    i, j, k, vals = oracle.find_peaks(d, np.zeros(d.shape, np.int8), 2, 0.3)
    tab, axes = ht.read_homeltab(julia_table_path)
    finder = ht.HaloFinder(12, tab, *axes)
    dev = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a), dtype=dt,
                                                       device="cuda")
    finder.bind_fields(dev(d), *[dev(e) for e in eta])
    npk = len(i)
    ones = lambda v, dt: dev(np.full(npk, v), dt)
    F = br.features(finder, dev(i, torch.int32), dev(j, torch.int32), dev(k, torch.int32),
                    ones(3.0, torch.float64), ones(12, torch.int32), ones(1.0, torch.float32),
                    ones(1.6, torch.float32), 1.0, peak_delta=dev(vals))
    P = br.predict(finder, model, F).cpu().numpy()
    assert np.isfinite(P).all()
    assert F.shape == (npk, 16)


def test_features_match_numpy(ht, finder):
    """The per-peak features (ht_bracket_features) against a numpy restatement, for peaks
    inside the tile (all 32 cells of the shells r^2 = 1..4 present: the unrolled path) and
    on its faces, edges and corners (out-of-tile cells left out of the shell means)."""
    br = ht.bracket
    rng = np.random.default_rng(21)
    n = 20
    d = rng.standard_normal((n, n, n)).astype(np.float32)      # [k][j][i], i fastest
    eta = [rng.standard_normal((n, n, n)).astype(np.float32) for _ in range(3)]
    dev = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a), dtype=dt,
                                                       device="cuda")
    finder.bind_fields(dev(d), *[dev(e) for e in eta])
    pts = [(i, j, k) for i in (1, 2, 3, 10, n - 1, n) for j in (1, 3, 11, n)
           for k in (1, 2, 9, n - 2, n)]
    pts += [tuple(int(x) for x in rng.integers(1, n + 1, 3)) for _ in range(200)]
    pi, pj, pk = (np.array([p[a] for p in pts], np.int32) for a in range(3))
    npk = len(pts)
    Rf = rng.uniform(1.5, 6.0, npk)
    ir2 = rng.integers(1, 30, npk).astype(np.int32)
    zz = rng.uniform(1.0, 2.0, npk).astype(np.float32)
    fc = rng.uniform(1.5, 1.8, npk).astype(np.float32)
    pd = rng.standard_normal(npk).astype(np.float32)
    alatt = 1.3
    F = br.features(finder, dev(pi, torch.int32), dev(pj, torch.int32), dev(pk, torch.int32),
                    dev(Rf, torch.float64), dev(ir2, torch.int32), dev(zz), dev(fc), alatt,
                    peak_delta=dev(pd)).cpu().numpy()
    r2 = finder.shell_r2().astype(np.int64)          # entry m - 1 is shell m
    ns = len(r2)
    offs = {s: [(a, b, c) for c in range(-2, 3) for b in range(-2, 3) for a in range(-2, 3)
                if a * a + b * b + c * c == s] for s in (1, 2, 3, 4)}
    want = np.zeros((npk, 16), np.float32)
    for q, (i, j, k) in enumerate(pts):
        want[q, 0] = Rf[q] / alatt
        want[q, 1] = np.sqrt(np.float32(ir2[q]))
        want[q, 2], want[q, 3], want[q, 4] = pd[q], fc[q], zz[q]
        want[q, 5] = d[k - 1, j - 1, i - 1]
        for s in (1, 2, 3, 4):
            v = [d[k - 1 + c, j - 1 + b, i - 1 + a] for a, b, c in offs[s]
                 if 1 <= i + a <= n and 1 <= j + b <= n and 1 <= k + c <= n]
            want[q, 5 + s] = np.sum(np.float64(v)) / len(v) if v else 0.0
        m0 = next((m for m in range(1, ns) if r2[m - 1] > ir2[q]), ns - 1)
        want[q, 10] = np.sqrt(float(r2[m0 - 1]))
        want[q, 11] = Rf[q] / alatt + 2.0
    np.testing.assert_allclose(F[:, :12], want[:, :12], rtol=2e-6, atol=2e-6)
    assert np.all(F[:, 12:] == 0)
