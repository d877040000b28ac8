"""Failure handling on the device path without a GPU fault: faults are injected on the host
side of the API (HT_FAULT_INJECT=alloc|launch makes the allocation or the dispatch fail
before the device is touched), every entry point must return HT_ERR_FAULT with a message
instead of exiting, and the context must stay usable once the injection stops.  On the
device, a bounded wait is made to run out (a TMA stage whose announced bytes never all
arrive): the kernel reports it through ht_device_status and the context stays usable."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

HT_ERR_FAULT = 6


@pytest.fixture
def inject(monkeypatch):
    def set_(v):
        if v:
            monkeypatch.setenv("HT_FAULT_INJECT", v)
        else:
            monkeypatch.delenv("HT_FAULT_INJECT", raising=False)
    yield set_
    monkeypatch.delenv("HT_FAULT_INJECT", raising=False)


def test_allocation_fault_on_create(ht, julia_table_path, inject):
    tab, axes = ht.read_homeltab(julia_table_path)
    inject("alloc")
    with pytest.raises(ht.HTError) as e:
        ht.HaloFinder(6, tab, *axes)
    assert e.value.code == HT_ERR_FAULT and "injected allocation fault" in str(e.value)
    inject(None)
    f = ht.HaloFinder(6, tab, *axes)      # the library recovers: a clean create succeeds
    assert f.nshells > 3


def test_launch_fault_then_recovery(ht, oracle, julia_table_path, inject):
    tab, axes = ht.read_homeltab(julia_table_path)
    finder = ht.HaloFinder(6, tab, *axes)
    n = 40
    rng = np.random.default_rng(0)
    d = rng.standard_normal((n, n, n)).astype(np.float32)
    dd = torch.as_tensor(d, device="cuda")
    mask = torch.zeros((n, n, n), dtype=torch.int8, device="cuda")
    out = ht.HaloFinder.alloc_peaks(1 << 16, "cuda", False)
    inject("launch")
    with pytest.raises(ht.HTError) as e:
        finder.peakfind_filter(dd, mask, 2, 0.5, 1, 1 << 16, out)
    assert e.value.code == HT_ERR_FAULT
    with pytest.raises(ht.HTError) as e:
        finder.bind_fields(dd, dd, dd, dd)
    assert e.value.code == HT_ERR_FAULT
    inject(None)
    finder.peakfind_filter(dd, mask, 2, 0.5, 1, 1 << 16, out)
    torch.cuda.synchronize()
    npk = int(out["count"].item())
    oi, oj, ok, _ = oracle.find_peaks(d, np.zeros(d.shape, np.int8), 2, 0.5)
    assert npk == len(oi) and list(out["i"][:npk].cpu().numpy()) == list(oi)
    assert finder.device_status() == 0


def test_bounded_wait_runs_out_then_recovers(ht, oracle, julia_table_path):
    """A bounded in-kernel wait that nothing completes, without a fault or a hang: with
    HT_TUNE_INJECT_TX every CTA of the TMA peak scan announces 16 bytes more than its
    first copy delivers, so that stage's mbarrier phase never completes although the copy
    lands.  With a 1 ms limit (HT_TUNE_WAIT_NS) each CTA gives up, records status 1,
    waits (bounded again) for its copies and returns; ht_device_status reports the
    timeout once and clears it.  With the hook off the same context scans the same field
    exactly as the oracle does."""
    import time
    tab, axes = ht.read_homeltab(julia_table_path)
    finder = ht.HaloFinder(6, tab, *axes)
    n, nbuff, fcrit = 64, 4, 1.5       # 256-byte rows: the scan takes the TMA path
    rng = np.random.default_rng(3)
    d = rng.standard_normal((n, n, n)).astype(np.float32)
    dd = torch.as_tensor(d, device="cuda")
    mask = torch.zeros((n, n, n), dtype=torch.int8, device="cuda")
    out = ht.HaloFinder.alloc_peaks(1 << 16, "cuda", False)
    assert finder.device_status() == 0
    finder.tune(wait_ns=1_000_000, inject_tx=16)
    t0 = time.perf_counter()
    finder.peakfind_filter(dd, mask, nbuff, fcrit, 1, 1 << 16, out)
    status = finder.device_status()          # synchronises
    elapsed = time.perf_counter() - t0
    assert status == 1, status
    assert elapsed < 5.0, elapsed            # the waits gave up after about 1 ms each
    assert finder.device_status() == 0       # read once, then cleared
    finder.tune(inject_tx=0, wait_ns=2_000_000_000)
    mask.zero_()
    out["count"].zero_()
    out["found"].zero_()
    finder.peakfind_filter(dd, mask, nbuff, fcrit, 1, 1 << 16, out)
    torch.cuda.synchronize()
    assert finder.device_status() == 0
    npk = int(out["count"].item())
    oi, oj, ok, od = oracle.find_peaks(d, np.zeros(d.shape, np.int8), nbuff, fcrit)
    assert npk == len(oi) > 0
    assert np.array_equal(out["i"][:npk].cpu().numpy(), oi)
    assert np.array_equal(out["j"][:npk].cpu().numpy(), oj)
    assert np.array_equal(out["k"][:npk].cpu().numpy(), ok)
    with pytest.raises(ht.HTError):
        finder.tune(inject_tx=8)             # not a multiple of 16
    with pytest.raises(ht.HTError):
        finder.tune(wait_ns=10)              # below the 1 us minimum
