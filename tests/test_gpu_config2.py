"""Parity at the plain-vs-batched workload's geometry (512^3 box, L = 1000 Mpc/h, 54-cell
wrap = 620^3 tile, 60 top-hat filters R = 1.5-60 Mpc/h, nhunt 53: 2,344 shells, above the
reference GPU kernel's 512-shell cap), seed 1: every peak of the tile (several million)
through the PLAIN, BATCHED and LEARNED walks must give bit-identical results and masks; a
random sample is compared with the FP64 oracle in both conventions (the reference GPU
entry and RadialShell.analyse_peak) under the tolerance of oracle/parity.py (1e-5
relative, widened by the reference's own Float32 rounding noise where that is larger;
flips only within 1e-6 of the barrier), and against the full-FP64 oracle at 1e-5."""
import numpy as np
import pytest
import torch

from gpu_helpers import make_box_workload, oracle_sample, print_report, result_rows

pytestmark = pytest.mark.gpu

N, L, NBUFF, NF, RMIN, RMAX, SEED = 512, 1000.0, 54, 60, 1.5, 60.0, 1
SAMPLE_GPU, SAMPLE_CPU = 3000, 800


@pytest.fixture(scope="module")
def box(ht):
    W = make_box_workload(ht, N, L, NBUFF, NF, RMIN, RMAX, SEED)
    yield W
    W["finder"].close()


def test_config2_modes_bit_identical(ht, box):
    W = box
    npk, finder, t = W["npk"], W["finder"], W["tile"]
    assert finder.nshells == 2344 and npk > 1_000_000
    finder.bind_fields(t["delta"], t["etax"], t["etay"], t["etaz"], t["eta2x"], t["eta2y"],
                       t["eta2z"], None)
    model = ht.bracket.BracketModel.load(device="cuda")
    F = ht.bracket.features(finder, *W["args"], peak_delta=W["peaks"]["delta"][:npk])
    cost = ht.bracket.predict(finder, model, F)[:, 1].contiguous()
    outs, masks = {}, {}
    for mode in ("plain", "batched", "learned"):
        mask = torch.zeros_like(t["delta"], dtype=torch.int8)
        outs[mode] = finder.analyse(*W["args"], nbuff=NBUFF, mask=mask, mode=mode,
                                    cost=cost if mode == "learned" else None)
        masks[mode] = mask
    torch.cuda.synchronize()
    for mode in ("batched", "learned"):
        for k in outs["plain"]:
            a, b = outs["plain"][k], outs[mode][k]
            assert torch.equal(a.view(torch.int32), b.view(torch.int32)), (mode, k)
        assert torch.equal(masks["plain"], masks[mode]), mode


@pytest.mark.parametrize("conv,kind,size", [("gpu", "cudakernel", SAMPLE_GPU),
                                            ("cpu", "radialshell", SAMPLE_CPU)])
def test_config2_vs_oracle(ht, oracle, box, conv, kind, size):
    from oracle import parity
    W = box
    npk, finder, t = W["npk"], W["finder"], W["tile"]
    finder.bind_fields(t["delta"], t["etax"], t["etay"], t["etaz"], t["eta2x"], t["eta2y"],
                       t["eta2z"], None)
    model = ht.bracket.BracketModel.load(device="cuda")
    F = ht.bracket.features(finder, *W["args"], peak_delta=W["peaks"]["delta"][:npk])
    cost = ht.bracket.predict(finder, model, F)[:, 1].contiguous()
    res = finder.analyse(*W["args"], nbuff=NBUFF, conv=conv, mode="learned", cost=cost)
    torch.cuda.synchronize()
    rng = np.random.default_rng(7 if conv == "gpu" else 8)
    sel = np.sort(rng.choice(npk, size=size, replace=False))
    ox, t_x = oracle_sample(oracle, W, sel, kind, exact_products=True)
    o, t_cpu = oracle_sample(oracle, W, sel, kind)
    rows = result_rows(ht, res, npk, sel)
    rep_x = parity.report(rows, ox)
    print_report(rep_x, f"config-2 {conv} convention vs full-FP64 oracle ({kind}, {t_x:.1f} s)")
    rep = parity.report(rows, o, ora_exact=ox)
    print_report(rep, f"config-2 {conv} convention vs reference-semantics oracle ({kind}, "
                      f"{t_cpu:.1f} s)")
    for rp in (rep_x, rep):
        assert rp["flips_unexplained"] == 0, rp["flip_list"]
        assert rp["mismatches"] == 0, rp["mismatch_list"]
    assert rep["collapsed"] > 0.3 * size
