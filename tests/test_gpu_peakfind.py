"""Peak finder on the GPU vs the CPU oracle (PeakFind.jl:15-78): bit-exact indices,
values, filter indices, order and mask, on the reference's known-answer cases and on
smoothed random fields with the mask carried across filters."""
import numpy as np
import pytest

from gpu_helpers import gpu_find_peaks

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def finder(ht, fortran_table_path):
    tab, axes = ht.read_homeltab(fortran_table_path)
    return ht.HaloFinder(4, tab, *axes)


def _cell(a, i, j, k, v):
    a[k - 1, j - 1, i - 1] = v


def _both(ht, oracle, finder, fields, nbuff, fcrits, max_peaks=1 << 20, mask=None,
          lapd=None):
    n = fields[0].shape[0]
    mask = np.zeros((n, n, n), np.int8) if mask is None else mask
    g, gmask = gpu_find_peaks(ht, finder, fields, mask.copy(), nbuff, fcrits, max_peaks,
                              lapd_s=lapd)
    om = mask.copy()
    oi, oj, ok, od, of = [], [], [], [], []
    left = max_peaks
    for fi, (ds, fc) in enumerate(zip(fields, fcrits), start=1):
        if left <= 0:
            break
        i, j, k, d = oracle.find_peaks(ds, om, nbuff, fc, left)
        oi += list(i); oj += list(j); ok += list(k); od += list(d); of += [fi] * len(i)
        left -= len(i)
    assert list(g["i"]) == oi and list(g["j"]) == oj and list(g["k"]) == ok
    assert np.array_equal(g["delta"].view(np.int32), np.asarray(od, np.float32).view(np.int32))
    assert list(g["filter_idx"]) == of
    assert np.array_equal(gmask, om)
    return g


def test_reference_kats(ht, oracle, finder):
    n = 11
    d = np.zeros((n, n, n), np.float32); _cell(d, 6, 6, 6, 2.0)
    g = _both(ht, oracle, finder, [d], 1, [1.0])
    assert list(zip(g["i"], g["j"], g["k"])) == [(6, 6, 6)]
    _both(ht, oracle, finder, [np.full((n, n, n), 0.5, np.float32)], 1, [1.0])
    grad = np.fromfunction(lambda k, j, i: i + j + k + 3.0, (n, n, n)).astype(np.float32)
    assert len(_both(ht, oracle, finder, [grad], 1, [1.0])["i"]) == 0
    m = np.zeros((n, n, n), np.int8); m[5, 5, 5] = 1
    assert len(_both(ht, oracle, finder, [d], 1, [1.0], mask=m)["i"]) == 0
    d2 = np.zeros((n, n, n), np.float32); _cell(d2, 1, 6, 6, 2.0)
    assert len(_both(ht, oracle, finder, [d2], 1, [1.0])["i"]) == 0
    n = 15
    d4 = np.zeros((n, n, n), np.float32)
    for c in [(4, 4, 4), (4, 4, 12), (12, 12, 4), (12, 12, 12)]:
        _cell(d4, *c, 2.0)
    g = _both(ht, oracle, finder, [d4], 1, [1.0], max_peaks=2)
    assert len(g["i"]) == 2


def _smooth_random(n, seed, radii):
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((n, n, n))
    wk = np.fft.rfftn(w)
    k = np.sqrt(np.add.outer(np.add.outer(np.fft.fftfreq(n) ** 2, np.fft.fftfreq(n) ** 2),
                             np.fft.rfftfreq(n) ** 2)) * 2 * np.pi
    out = []
    for R in radii:
        x = k * R
        with np.errstate(invalid="ignore", divide="ignore"):
            win = np.where(x == 0, 1.0, 3 * (np.sin(x) - x * np.cos(x)) / x ** 3)
        f = np.fft.irfftn(wk * win, s=(n, n, n))
        out.append((f / f.std()).astype(np.float32))
    return out


# n % 4 == 0 and n >= 40 take the TMA plane ring (48, 64, 132, 136); the others the
# plain-load ring.  132 and 136 span several k-chunks per column.
@pytest.mark.parametrize("n,nbuff", [(48, 4), (45, 3), (70, 1), (37, 5), (64, 1), (132, 2),
                                     (136, 4)])
def test_random_fields_mask_carried(ht, oracle, finder, n, nbuff):
    fields = _smooth_random(n, n + nbuff, [4.0, 2.5, 1.5, 1.0])
    g = _both(ht, oracle, finder, fields, nbuff, [1.0, 1.2, 0.5, 0.0])
    assert len(g["i"]) > 20


def test_nan_cells(ht, oracle, finder):
    """NaN neighbours never reject a peak, and a NaN centre is a peak unless masked:
    `ff < fcrit` and `neighbour > ff` are both false when NaN is involved
    (PeakFind.jl:40-60)."""
    for n in (40, 41):
        f = _smooth_random(n, 9, [1.5])[0]
        rng = np.random.default_rng(n)
        idx = tuple(rng.integers(0, n, size=(3, 60)))
        f[idx] = np.nan
        _both(ht, oracle, finder, [f], 2, [0.3])
    assert finder.device_status() == 0


def test_truncation_across_filters(ht, oracle, finder):
    fields = _smooth_random(40, 1, [2.0, 1.0])
    total = len(_both(ht, oracle, finder, fields, 2, [0.0, 0.0])["i"])
    for mp in (1, 7, total // 2, total - 1):
        g = _both(ht, oracle, finder, fields, 2, [0.0, 0.0], max_peaks=mp)
        assert len(g["i"]) == mp


def test_ties_and_plateaus(ht, oracle, finder):
    n = 20
    d = np.zeros((n, n, n), np.float32)
    d[5:8, 5:8, 5:8] = 3.0          # a plateau: every cell of it is a peak (ties pass)
    d[12, 12, 12] = 2.0; d[12, 12, 13] = 2.0
    g = _both(ht, oracle, finder, [d], 2, [1.0])
    assert len(g["i"]) == 27 + 2


def test_lapd_sampled_at_peaks(ht, oracle, finder):
    fields = _smooth_random(32, 5, [2.0])
    lap = _smooth_random(32, 6, [1.0])
    g = _both(ht, oracle, finder, fields, 2, [0.5], lapd=lap)
    idx = (g["k"] - 1, g["j"] - 1, g["i"] - 1)
    assert np.array_equal(g["lapd"], lap[0][idx])


@pytest.mark.parametrize("wsmooth", [0, 1, 3])
def test_smoothing_window(ht, finder, wsmooth):
    """ht_smooth_window vs the FP64 window of Filters.smooth_field (Filters.jl:72-99)."""
    import torch
    n, box, Rf = 24, 60.0, 7.5
    rng = np.random.default_rng(wsmooth)
    a = rng.standard_normal((n, n, n)).astype(np.float32)
    ak = np.fft.rfftn(a).astype(np.complex64)
    dk = 2 * np.pi / box
    kz = np.fft.fftfreq(n, 1.0 / n) * dk
    kx = np.arange(n // 2 + 1) * dk
    k2 = kz[:, None, None] ** 2 + kz[None, :, None] ** 2 + kx[None, None, :] ** 2
    k = np.sqrt(k2)
    x = k * Rf
    with np.errstate(invalid="ignore", divide="ignore"):
        if wsmooth == 0:
            w = np.exp(-x * x / 8)
        elif wsmooth == 3:
            w = np.exp(-x * x / 8) * k2
        else:
            w = 3 * (np.sin(x) - x * np.cos(x)) / x ** 3
    w = np.where(k2 == 0, 1.0, w).astype(np.float32)
    ref = ak * w
    got = finder.smooth_window(torch.as_tensor(ak, device="cuda"), n, box, Rf, wsmooth)
    got = got.cpu().numpy()
    assert np.allclose(got, ref, rtol=1e-6, atol=1e-6 * np.abs(ref).max())
    assert got[0, 0, 0] == ak[0, 0, 0]


def test_smooth_box_wrapped_matches_torch(ht, finder):
    """ht_smooth_filter (window + cuFFT C2R + periodic wrap) vs torch irfftn + wrap."""
    import torch
    import torch.nn.functional as F
    n, nb, box, Rf = 32, 5, 80.0, 6.0
    rng = np.random.default_rng(9)
    a = torch.as_tensor(rng.standard_normal((n, n, n)).astype(np.float32), device="cuda")
    ak = torch.fft.rfftn(a, dim=(0, 1, 2)).contiguous()
    got = finder.smooth_box_wrapped(ak, n, nb, box, Rf, 1)
    w = finder.smooth_window(ak, n, box, Rf, 1)
    ref = torch.fft.irfftn(w, s=(n, n, n), dim=(0, 1, 2))
    ref = F.pad(ref[None, None], (nb,) * 6, mode="circular")[0, 0]
    torch.cuda.synchronize()
    assert got.shape == ref.shape
    assert torch.allclose(got, ref, rtol=1e-5, atol=1e-6 * float(ref.abs().max()))


@pytest.mark.parametrize("n,wsmooth,path", [(36, 1, 0), (40, 0, 0), (30, 3, 0), (32, 1, 0),
                                            (36, 1, 1), (32, 1, 2), (44, 0, 2)])
def test_smooth_tile_matches_fp64(ht, finder, n, wsmooth, path):
    """ht_smooth_tile vs numpy FP64 irfftn of the FP64-windowed rfft: the tile smoothing of
    peak_find_tile_gpu (ext/CUDAExt.jl:2951-2989), boxsize = n * alatt.  path 0 picks by
    size (3-D cuFFT plan for powers of two, transposes + batched 1-D transforms for other
    even sides); 1 and 2 force one of them."""
    import torch
    finder.tune(fft_path=path)
    try:
        _check_smooth_tile(finder, n, wsmooth)
    finally:
        finder.tune(fft_path=0)


def _check_smooth_tile(finder, n, wsmooth):
    import torch
    alatt, Rf = 1.9, 5.0
    box = n * alatt
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n, n)).astype(np.float32)
    ak = torch.fft.rfftn(torch.as_tensor(a, device="cuda"), dim=(0, 1, 2)).contiguous()
    got = finder.smooth_tile(ak, n, box, Rf, wsmooth).cpu().numpy()
    akh = ak.cpu().numpy().astype(np.complex128)
    dk = 2 * np.pi / box
    kz = np.fft.fftfreq(n, 1.0 / n) * dk
    kx = np.arange(n // 2 + 1) * dk
    k2 = kz[:, None, None] ** 2 + kz[None, :, None] ** 2 + kx[None, None, :] ** 2
    x = np.sqrt(k2) * Rf
    with np.errstate(invalid="ignore", divide="ignore"):
        w = {0: np.exp(-x * x / 8), 3: np.exp(-x * x / 8) * k2}.get(
            wsmooth, 3 * (np.sin(x) - x * np.cos(x)) / x ** 3)
    w = np.where(k2 == 0, 1.0, w)
    ref = np.fft.irfftn(akh * w, s=(n, n, n))
    scale = np.abs(ref).max()
    assert got.shape == (n, n, n) and got.dtype == np.float32
    # FP32 FFT round-off: a few ulp of the field's range
    assert np.abs(got - ref).max() <= 2e-6 * scale * np.log2(n ** 3)


@pytest.mark.parametrize("n", [576, 1152])
def test_fused_fft_matches_transposed_path(ht, finder, n):
    """The fused three-pass inverse FFT (warp-level FFTs in shared memory, sides 576 and
    1152) against the transposed cuFFT path (itself checked against FP64 above): the same
    transform up to FP32 round-off."""
    import torch
    rng = np.random.default_rng(n)
    a = torch.as_tensor(rng.standard_normal((n, n, n)).astype(np.float32), device="cuda")
    ak = torch.fft.rfftn(a, dim=(0, 1, 2)).contiguous()
    del a
    outs = []
    try:
        for path in (2, 3):
            finder.tune(fft_path=path)
            outs.append(finder.smooth_tile(ak, n, n * 1.46, 6.0, 1).cpu().numpy())
    finally:
        finder.tune(fft_path=0)
    ref, got = outs
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 2e-6 * scale * np.log2(n ** 3)
    assert finder.device_status() == 0


@pytest.mark.parametrize("n,wsmooth", [(576, 1), (576, 0), (576, 3), (1152, 1)])
def test_pencil_fft_matches_transposed_path(ht, finder, n, wsmooth):
    """The pencil passes (spectrum transposed once to kz-contiguous pencils, then window +
    FFT along kz, FFT along ky, half-length real FFT along kx, each pass reading whole
    columns) against the transposed cuFFT path (itself checked against FP64 above), both
    as ht_smooth_pencil on the full range and as ht_smooth_tile's path 4."""
    import torch
    rng = np.random.default_rng(n + wsmooth)
    a = torch.as_tensor(rng.standard_normal((n, n, n)).astype(np.float32), device="cuda")
    ak = torch.fft.rfftn(a, dim=(0, 1, 2)).contiguous()
    del a
    box, Rf = n * 1.46, 6.0
    try:
        finder.tune(fft_path=2)
        ref = finder.smooth_tile(ak, n, box, Rf, wsmooth)
        finder.tune(fft_path=4)
        via_tile = finder.smooth_tile(ak, n, box, Rf, wsmooth)
    finally:
        finder.tune(fft_path=0)
    pk = finder.spectrum_pencil(ak, n)
    got = finder.smooth_pencil(pk, n, box, Rf, wsmooth, 0, n)
    torch.cuda.synchronize()
    scale = float(ref.abs().max())
    tol = 2e-6 * scale * np.log2(n ** 3)
    assert float((got - ref).abs().max()) <= tol
    assert torch.equal(got, via_tile)      # same kernels, same order: bit-identical
    assert finder.device_status() == 0


@pytest.mark.parametrize("n,lo,hi", [(576, 63, 513), (1152, 63, 1089)])
def test_pencil_region_rows(ht, finder, n, lo, hi):
    """ht_smooth_pencil(lo, hi) writes exactly the rows (z, y) in [lo, hi)^2, equal to the
    full transform's, and leaves every other row of the output untouched."""
    import torch
    rng = np.random.default_rng(hi)
    a = torch.as_tensor(rng.standard_normal((n, n, n)).astype(np.float32), device="cuda")
    ak = torch.fft.rfftn(a, dim=(0, 1, 2)).contiguous()
    del a
    pk = finder.spectrum_pencil(ak, n)
    del ak
    full = finder.smooth_pencil(pk, n, n * 1.9, 4.0, 1, 0, n)
    part = torch.full((n, n, n), float("nan"), device="cuda")
    finder.smooth_pencil(pk, n, n * 1.9, 4.0, 1, lo, hi, out=part)
    torch.cuda.synchronize()
    assert torch.equal(part[lo:hi, lo:hi], full[lo:hi, lo:hi])
    written = ~torch.isnan(part).all(dim=2)
    expect = torch.zeros((n, n), dtype=torch.bool, device="cuda")
    expect[lo:hi, lo:hi] = True
    assert torch.equal(written, expect)
    assert not torch.isnan(part[lo:hi, lo:hi]).any()


def test_pencil_rejects_bad_arguments(ht, finder):
    import torch
    assert ht.HaloFinder.pencil_supported(576) and ht.HaloFinder.pencil_supported(1152)
    assert not ht.HaloFinder.pencil_supported(620)
    pk = torch.zeros((4, 3, 4), dtype=torch.complex64, device="cuda")
    with pytest.raises(ValueError):
        finder.smooth_pencil(pk, 576, 100.0, 4.0, 1, 0, 576)
    big = torch.zeros((2, 2, 2), dtype=torch.complex64, device="cuda")
    with pytest.raises(ht.HTError):   # side 620 has no pencil passes: reported, not run
        ht._lib.check(ht._lib.load().ht_smooth_pencil(finder.handle, big.data_ptr(),
                                                      big.data_ptr(), 620, 100.0, 4.0, 1, 0,
                                                      620, None))


@pytest.mark.parametrize("n,lo,hi", [(44, 3, 41), (620, 53, 567)])
def test_smooth_tile_planes(ht, finder, n, lo, hi):
    """ht_smooth_tile_planes delivers planes [lo, hi) equal to the full transform's."""
    import torch
    rng = np.random.default_rng(lo)
    a = torch.as_tensor(rng.standard_normal((n, n, n)).astype(np.float32), device="cuda")
    ak = torch.fft.rfftn(a, dim=(0, 1, 2)).contiguous()
    full = finder.smooth_tile(ak, n, n * 1.9, 4.0, 1).cpu().numpy()
    part = torch.full((n, n, n), float("nan"), device="cuda")
    finder.smooth_tile(ak, n, n * 1.9, 4.0, 1, out=part, planes=(lo, hi))
    part = part.cpu().numpy()
    scale = np.abs(full).max()
    assert np.abs(part[lo:hi] - full[lo:hi]).max() <= 1e-6 * scale

