"""Parity at the large tile's shell geometry: the headline workload's cell size and hunt
radius (alatt 1.4648 Mpc/h, nbuff 64, nhunt 63: 3,310 shells, six times the reference GPU
kernel's 512-shell cap) on a 192^3 periodic box wrapped to a 320^3 tile, 80 top-hat filters
R = 1.5-80 Mpc/h, seed 5.  Every peak of the tile through the PLAIN, BATCHED and LEARNED
walks gives bit-identical results and masks; random samples are compared with the FP64
oracle in both conventions (the reference GPU entry and RadialShell.analyse_peak) under the
rule of oracle/parity.py (1e-5 relative, widened by the reference's own Float32 rounding
noise where that is larger; flips only within 1e-6 of the barrier) and with the full-FP64
oracle at 1e-5."""
import numpy as np
import pytest
import torch

from gpu_helpers import make_box_workload, oracle_sample, print_report, result_rows

pytestmark = pytest.mark.gpu

N, L, NBUFF, NF, RMIN, RMAX, SEED = 192, 281.25, 64, 80, 1.5, 80.0, 5
SAMPLE_GPU, SAMPLE_CPU = 3000, 600


@pytest.fixture(scope="module")
def tile(ht):
    W = make_box_workload(ht, N, L, NBUFF, NF, RMIN, RMAX, SEED)
    yield W
    W["finder"].close()


def _cost(ht, W):
    finder = W["finder"]
    model = ht.bracket.BracketModel.load(device="cuda")
    F = ht.bracket.features(finder, *W["args"], peak_delta=W["peaks"]["delta"][:W["npk"]])
    return ht.bracket.predict(finder, model, F)[:, 1].contiguous()


def _bind(W):
    t = W["tile"]
    W["finder"].bind_fields(t["delta"], t["etax"], t["etay"], t["etaz"], t["eta2x"],
                            t["eta2y"], t["eta2z"], None)


def test_tile_geometry_modes_bit_identical(ht, tile):
    W = tile
    npk, finder = W["npk"], W["finder"]
    assert finder.nhunt == 63 and finder.nshells == 3310 and npk > 50_000
    _bind(W)
    cost = _cost(ht, W)
    outs, masks = {}, {}
    for mode in ("plain", "batched", "learned"):
        mask = torch.zeros_like(W["tile"]["delta"], dtype=torch.int8)
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
def test_tile_geometry_vs_oracle(ht, oracle, tile, conv, kind, size):
    from oracle import parity
    W = tile
    npk, finder = W["npk"], W["finder"]
    _bind(W)
    res = finder.analyse(*W["args"], nbuff=NBUFF, conv=conv, mode="learned", cost=_cost(ht, W))
    torch.cuda.synchronize()
    rng = np.random.default_rng(11 if conv == "gpu" else 12)
    sel = np.sort(rng.choice(npk, size=min(size, npk), replace=False))
    ox, t_x = oracle_sample(oracle, W, sel, kind, exact_products=True)
    o, t_cpu = oracle_sample(oracle, W, sel, kind)
    rows = result_rows(ht, res, npk, sel)
    rep_x = parity.report(rows, ox)
    print_report(rep_x, f"nhunt-63 {conv} convention vs full-FP64 oracle ({kind}, {t_x:.1f} s)")
    rep = parity.report(rows, o, ora_exact=ox)
    print_report(rep, f"nhunt-63 {conv} convention vs reference-semantics oracle ({kind}, "
                      f"{t_cpu:.1f} s)")
    for rp in (rep_x, rep):
        assert rp["flips_unexplained"] == 0, rp["flip_list"]
        assert rp["mismatches"] == 0, rp["mismatch_list"]
    assert rep["collapsed"] > 0.3 * len(sel)
