"""Precision study on the small periodic-box workload (128^3 box, L = 250 Mpc/h, 36-cell
wrap, 30 top-hat filters R = 2-40 Mpc/h, nhunt 35, 1,024 shells): the device path (FP32
fields, per-lane FP64 shell sums with exact FP64 products, lanes combined in FP64 in a
fixed order, FP64 profile recurrence, eigen solve and barrier interpolation) against the
CPU oracle, which accumulates every sum in FP64 from the same FP32 fields in cell order
(RadialShell.jl:362-446 semantics).  The remaining differences are summation order, the
reference's Float32 rounding of each cell product (the oracle keeps it, the device forms
the products exactly) and the FP32 rounding of the outputs.

Two oracles.  The full-FP64 oracle forms every cell product exactly, as the device does:
against it every output field agrees to 1e-5 relative to its magnitude (e_v and p_v,
ratios of eigenvalue differences to the strain trace, to 1e-5 relative plus 1e-12 kappa,
kappa = max|eig| / |trace|, 500x the FP64 cancellation floor of the ratio).  The
reference-semantics oracle rounds each product to Float32 as Huntian.jl does: against it
the same 1e-5 applies, widened per peak and field by twice the reference's own rounding
noise (the difference of the two oracles), which p_v near zero amplifies.  A collapse flip
is allowed only where the oracle's decision margin (the smallest |Fbar - fcrit| or
|zvir - ZZon| of the comparisons that decided the collapse) is below 1e-6; every flip is
listed.  Both conventions: the reference GPU entry (every peak) and
RadialShell.analyse_peak (a random sample: the CPU convention walks every shell).  Run
with `-s` to print the error tables (oracle/parity.py)."""
import numpy as np
import pytest
import torch

from gpu_helpers import make_box_workload, oracle_sample, print_report, result_rows

pytestmark = pytest.mark.gpu

N, L, NBUFF, NF, RMIN, RMAX, SEED = 128, 250.0, 36, 30, 2.0, 40.0, 12345
SAMPLE = 50000      # every peak of the workload (about 43,000)
SAMPLE_CPU = 6000   # RadialShell.analyse_peak walks all 1,024 shells of every peak


def test_precision_vs_fp64_oracle(ht, oracle):
    from oracle import parity
    W = make_box_workload(ht, N, L, NBUFF, NF, RMIN, RMAX, SEED)
    npk = W["npk"]
    assert npk > 5000
    t = W["tile"]
    finder = W["finder"]
    finder.bind_fields(t["delta"], t["etax"], t["etay"], t["etaz"], t["eta2x"], t["eta2y"],
                       t["eta2z"], None)
    res = finder.analyse(*W["args"], nbuff=NBUFF)
    res_cpu = finder.analyse(*W["args"], nbuff=NBUFF, conv="cpu")
    torch.cuda.synchronize()
    rng = np.random.default_rng(0)
    for conv, kind, size, r in (("gpu", "cudakernel", SAMPLE, res),
                                ("cpu", "radialshell", SAMPLE_CPU, res_cpu)):
        sel = np.sort(rng.choice(npk, size=min(size, npk), replace=False))
        ox, t_x = oracle_sample(oracle, W, sel, kind, exact_products=True)
        o, t_cpu = oracle_sample(oracle, W, sel, kind)
        rows = result_rows(ht, r, npk, sel)
        rep_x = parity.report(rows, ox)
        print_report(rep_x, f"{conv} convention vs full-FP64 oracle ({kind}, {t_x:.1f} s)")
        rep = parity.report(rows, o, ora_exact=ox)
        print_report(rep, f"{conv} convention vs reference-semantics oracle ({kind}, "
                          f"{t_cpu:.1f} s)")
        for rp in (rep_x, rep):
            assert rp["flips_unexplained"] == 0, rp["flip_list"]
            assert rp["mismatches"] == 0, rp["mismatch_list"]
        assert rep_x["within_reference_noise"] == 0
        assert rep["collapsed"] > 0.5 * len(sel)
