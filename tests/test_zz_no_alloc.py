"""The allocation-free shell collapse, ht_shell_analyse_static.

Callers that cannot allocate device memory while they run this step (work issued into
a stream under CUDA-graph capture, or a host that owns the device memory pool) use
ht_shell_analyse_static, which keeps its scratch in a static array of the library.  It
must give the same results as ht_shell_analyse, bit for bit (both run the same walk over
the fields in place), on two calls in a row (the static array keeps the previous call's
contents); its results must agree with the oracle (oracle/parity.py), and the second call
must leave the device's free memory unchanged (the first call of a process may load the
library's device code and array).  This file is collected last on purpose.
"""
import numpy as np
import pytest
import torch

from gpu_helpers import to_dev

pytestmark = pytest.mark.gpu


def _case(seed, n=48):
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*(np.arange(1, n + 1),) * 3, indexing="ij")
    d = 0.1 * rng.standard_normal((n, n, n))
    for _ in range(25):
        c = rng.integers(6, n - 5, 3)
        d += (1.5 + 2.0 * rng.random()) * np.exp(
            -((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (8.0 + 20.0 * rng.random()))
    d = d.astype(np.float32)
    eta = [(0.3 * rng.standard_normal(d.shape)).astype(np.float32) for _ in range(6)]
    lapd = (0.05 * rng.standard_normal(d.shape)).astype(np.float32)
    return d, eta, lapd


def test_static_scratch_matches_allocating_entry(ht, oracle, julia_table_path):
    tab, axes = ht.read_homeltab(julia_table_path)
    finder = ht.HaloFinder(12, tab, *axes)
    for call, seed in enumerate((21, 22)):          # two calls in a row, different inputs
        d, eta, lapd = _case(seed)
        i, j, k, _ = oracle.find_peaks(d, np.zeros(d.shape, np.int8), 2, 0.6)
        npk = len(i)
        assert npk > 10
        fields = {"delta": to_dev(d), "etax": to_dev(eta[0]), "etay": to_dev(eta[1]),
                  "etaz": to_dev(eta[2]), "eta2x": to_dev(eta[3]), "eta2y": to_dev(eta[4]),
                  "eta2z": to_dev(eta[5]), "lapd": to_dev(lapd)}
        col = lambda v, dt: to_dev(np.broadcast_to(np.asarray(v), (npk,)), dt)
        args = (col(i, torch.int32), col(j, torch.int32), col(k, torch.int32),
                col(3.0, torch.float64), col(12, torch.int32), col(1.0, torch.float32),
                col(1.3, torch.float32), 1.5)
        finder.bind_fields(fields["delta"], fields["etax"], fields["etay"], fields["etaz"],
                           fields["eta2x"], fields["eta2y"], fields["eta2z"], fields["lapd"])
        mask_a = torch.zeros(d.shape, dtype=torch.int8, device="cuda")
        ref = finder.analyse(*args, nbuff=2, mask=mask_a, mode="batched")
        mask_b = torch.zeros(d.shape, dtype=torch.int8, device="cuda")
        out = ht.HaloFinder.alloc_results(npk, "cuda")
        for v in out.values():
            v.fill_(float("nan"))
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        finder.analyse_static(fields, *args, nbuff=2, mask=mask_b, out=out)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        if call == 1:
            assert free1 == free0, (free0, free1)
        for name in ht.RESULT_NAMES:
            w = ht.RESULT_WIDTH.get(name, 1)
            a = ref[name][:npk * w].view(torch.int32)
            b = out[name][:npk * w].view(torch.int32)
            assert torch.equal(a, b), (call, name)
        assert torch.equal(mask_a, mask_b), call
        assert (ref["RTHL"][:npk] > 0).any()
        # and the oracle (the reference's GPU-entry semantics, full-FP64 noise reference)
        from oracle import parity
        F = oracle.Fields(d, *eta[:3], *eta[3:], lapd=lapd)
        kw = dict(nbuff=2, kind="cudakernel")
        shells = oracle.precompute_shells(12)
        ct = oracle.read_homeltab(julia_table_path)
        ora_args = (F, i, j, k, 12, 3.0, 1.0, np.float32(1.3), 1.5, ct, shells)
        ox, _ = oracle.analyse_batch(*ora_args, exact_products=True, **kw)
        o, _ = oracle.analyse_batch(*ora_args, **kw)
        g = {n: out[n][:npk * ht.RESULT_WIDTH.get(n, 1)].cpu().numpy()
             .reshape(npk, -1) for n in ht.RESULT_NAMES}
        rep = parity.report(g, o, ora_exact=ox)
        assert rep["mismatches"] == 0 and rep["flips_unexplained"] == 0, rep
    finder.close()
