"""The learned walk bracket on held-out data: the plain-vs-batched geometry (512^3 box,
L = 1000 Mpc/h, 54-cell wrap, 60 filters R = 1.5-60 Mpc/h) at seed 9, which the shipped
weights (trained on seeds 1-8) never saw.

- hit rate: the fraction of peaks whose walk stops at a radius inside the predicted
  [low, high] quantile bracket;
- what the prediction buys: a warp walks the four peaks of a work item (8 lanes each)
  side by side and is held by the longest of the four, so the LEARNED order sorts the
  peaks of each spatial block by predicted walk length.  The lane efficiency of an order
  is the walked cells of its peaks over 4 x the cells of the longest walk in each item of
  4 consecutive peaks.  It is computed for the batch order (PLAIN), the Morton order
  (BATCHED), blocks sorted by the data-independent minimum walk, blocks sorted by the
  learned prediction (LEARNED's order) and blocks sorted by the true walk lengths (the
  best an order of this kind can do).  Run with -s to print the numbers."""
import numpy as np
import pytest
import torch

from gpu_helpers import make_box_workload

pytestmark = pytest.mark.gpu

BLOCK_BITS = 17
ITEM = 4   # peaks per warp (groups of 8 lanes)


def _spread3(v):
    x = v.astype(np.uint64) & np.uint64(0xFFFFF)
    for s, m in ((32, 0x1f00000000ffff), (16, 0x1f0000ff0000ff), (8, 0x100f00f00f00f00f),
                 (4, 0x10c30c30c30c30c3), (2, 0x1249249249249249)):
        x = (x | (x << np.uint64(s))) & np.uint64(m)
    return x


def _lane_efficiency(order, cells):
    c = cells[order]
    n = len(c) // ITEM * ITEM
    w = c[:n].reshape(-1, ITEM)
    return float(w.sum() / (ITEM * w.max(1).sum()))


def test_bracket_holdout_seed9(ht):
    W = make_box_workload(ht, 512, 1000.0, 54, 60, 1.5, 60.0, 9)
    npk, finder, t = W["npk"], W["finder"], W["tile"]
    finder.bind_fields(t["delta"], t["etax"], t["etay"], t["etaz"], t["eta2x"], t["eta2y"],
                       t["eta2z"], None)
    out = ht.HaloFinder.alloc_results(npk, "cuda", diagnostics=True)
    finder.analyse(*W["args"], nbuff=54, mode="batched", out=out)
    model = ht.bracket.BracketModel.load(device="cuda")
    F = ht.bracket.features(finder, *W["args"], peak_delta=W["peaks"]["delta"][:npk])
    pred = ht.bracket.predict(finder, model, F).cpu().numpy()
    torch.cuda.synchronize()
    ws = out["walk_shells"][:npk].cpu().numpy().astype(np.int64)
    r2 = finder.shell_r2().astype(np.float64)
    rad = np.sqrt(r2)
    true_r = rad[np.clip(ws, 1, len(rad)) - 1]
    hit = float(np.mean((pred[:, 0] <= true_r) & (true_r <= pred[:, 1])))
    below = float(np.mean(true_r < pred[:, 0]))
    above = float(np.mean(true_r > pred[:, 1]))

    # cells walked per peak (the cell table's cumulative counts up to the stop shell)
    nh = finder.nhunt
    g = np.arange(-nh, nh + 1)
    dz, dy, dx = np.meshgrid(g, g, g, indexing="ij")
    rr = (dx * dx + dy * dy + dz * dz).ravel()
    rr = rr[rr <= nh * nh]
    cum = np.cumsum(np.bincount(np.searchsorted(r2.astype(np.int64), rr), minlength=len(r2)))
    cells = cum[np.clip(ws, 1, len(r2)) - 1].astype(np.float64)

    # the data-independent minimum walk of each peak's filter: to the first shell past
    # rad[m0_init] + 2, m0_init the first shell past ir2min
    ir2 = W["ir2_all"].cpu().numpy()[W["fidx"].cpu().numpy()]
    m0i = np.clip(np.searchsorted(r2, ir2, side="right") + 1, 2, len(r2) - 1)
    smin_r = rad[np.clip(np.searchsorted(rad, rad[m0i - 1] + 2.0, side="right"), 0,
                         len(rad) - 1)]
    p = W["peaks"]
    i, j, k = (p[c][:npk].cpu().numpy().astype(np.int64) - 1 for c in ("i", "j", "k"))
    mort = _spread3(i) | (_spread3(j) << np.uint64(1)) | (_spread3(k) << np.uint64(2))
    blk = (mort >> np.uint64(BLOCK_BITS)).astype(np.int64)
    order_of = lambda length: np.lexsort((-np.floor(16.0 * length), blk))
    eff = {"batch order (PLAIN)": _lane_efficiency(np.arange(npk), cells),
           "Morton order (BATCHED)": _lane_efficiency(np.argsort(mort, kind="stable"), cells),
           "blocks, data-independent bound": _lane_efficiency(order_of(smin_r), cells),
           "blocks, learned (LEARNED)": _lane_efficiency(order_of(pred[:, 1]), cells),
           "blocks, true walk length": _lane_efficiency(order_of(true_r), cells)}
    print(f"\nseed 9 (held out): {npk} peaks, bracket hit rate {hit:.3f} "
          f"(below {below:.3f}, above {above:.3f})")
    for name, e in eff.items():
        print(f"lane efficiency, {name:32s} {e:.3f}")
    assert hit > 0.5
    assert eff["blocks, learned (LEARNED)"] > eff["Morton order (BATCHED)"]
    assert eff["blocks, learned (LEARNED)"] >= eff["blocks, data-independent bound"]
    finder.close()
