"""Reject-reason counters of the shell collapse (RadialShell.jl:13-32: premask, no_fcrit,
m0_one, no_collapse, rthl_neg) kept on the device, against the oracle's per-peak reject
codes on the small periodic-box workload (128^3 box, L = 250 Mpc/h, 36-cell wrap, 30
top-hat filters R = 2-40 Mpc/h, nhunt 35): every peak in the reference GPU convention, a
random sample in the RadialShell.analyse_peak convention.  A count may differ from the
oracle's by at most the number of collapse flips (peaks whose decision lies within 1e-6 of
a barrier, which the parity rule allows); the counters add up across calls until reset.
Run with -s to print the counts."""
import numpy as np
import pytest
import torch

from gpu_helpers import make_box_workload, oracle_sample, result_rows

pytestmark = pytest.mark.gpu

N, L, NBUFF, NF, RMIN, RMAX, SEED = 128, 250.0, 36, 30, 2.0, 40.0, 12345
ORACLE_CODE = {"premask": 1, "no_fcrit": 2, "m0_one": 3, "no_collapse": 4, "rthl_neg": 5}


def _subset(W, sel):
    idx = torch.as_tensor(sel, dtype=torch.long, device="cuda")
    return tuple(a[idx] if isinstance(a, torch.Tensor) else a for a in W["args"])


def _compare(ht, oracle, W, sel, conv, kind):
    from oracle import parity
    finder = W["finder"]
    finder.reset_reject_counts()
    res = finder.analyse(*_subset(W, sel), nbuff=NBUFF, conv=conv)
    got = finder.reject_counts()
    o, _, codes = oracle_sample(oracle, W, sel, kind, with_codes=True)
    rows = result_rows(ht, res, len(sel), np.arange(len(sel)))
    rep = parity.report(rows, o)
    want = {k: int((codes == c).sum()) for k, c in ORACLE_CODE.items()}
    print(f"\n{conv} convention, {len(sel)} peaks: device {got}, oracle {want}, "
          f"flips {rep['flips']}")
    collapsed = int((rows["RTHL"][:, 0] > 0).sum())
    assert sum(got.values()) == len(sel) - collapsed
    assert got["outside"] == 0 and got["premask"] == 0
    for k in ORACLE_CODE:
        assert abs(got[k] - want[k]) <= rep["flips"], (k, got, want)
    assert sum(want.values()) > 0
    return got


def test_reject_counts_match_oracle(ht, oracle):
    W = make_box_workload(ht, N, L, NBUFF, NF, RMIN, RMAX, SEED)
    npk = W["npk"]
    t = W["tile"]
    finder = W["finder"]
    finder.bind_fields(t["delta"], t["etax"], t["etay"], t["etaz"], t["eta2x"], t["eta2y"],
                       t["eta2z"], None)
    rng = np.random.default_rng(3)
    every = np.arange(npk)
    got = _compare(ht, oracle, W, every, "gpu", "cudakernel")
    sample = np.sort(rng.choice(npk, size=min(2000, npk), replace=False))
    _compare(ht, oracle, W, sample, "cpu", "radialshell")

    # the counters add up across calls until reset, in every mode
    finder.reset_reject_counts()
    for mode in ("plain", "batched"):
        finder.analyse(*W["args"], nbuff=NBUFF, mode=mode)
    twice = finder.reject_counts()
    assert twice == {k: 2 * v for k, v in got.items()}
    finder.reset_reject_counts()
    torch.cuda.synchronize()
    assert all(v == 0 for v in finder.reject_counts().values())
    finder.close()
