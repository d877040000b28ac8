"""Failure handling on the device path without a GPU fault: faults are injected on the host
side of the API (HT_FAULT_INJECT=alloc|launch makes the allocation or the dispatch fail
before the device is touched), every entry point must return HT_ERR_FAULT with a message
instead of exiting, and the context must stay usable once the injection stops."""
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
