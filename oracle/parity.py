"""Parity report of device results against oracle results -- TEST INFRASTRUCTURE ONLY.

Used by tests/ and by bench.py's CPU-baseline leg to state how the library's shell
collapse agrees with the FP64 restatement of the reference on the same peaks:

- collapse flips: peaks that collapse in one and not the other.  A flip is allowed only
  where the oracle's decision margin (the smallest |Fbar - fcrit| or |zvir - ZZon| of the
  comparisons that decided the collapse, ``margin`` in the oracle result) is below
  ``flip_margin`` (1e-6);
- mismatches: on peaks that collapse in both, any output field whose error exceeds
  ``rel`` (1e-5) relative to the field's magnitude (vectors and the strain matrix: their
  largest component).  e_v and p_v are ratios of eigenvalue differences to the strain
  trace; with kappa = max|eig| / |trace| of the final strain, an FP64 evaluation of them
  carries an absolute cancellation error of order 1e-15 kappa, so their tolerance is
  ``rel * |x| + 1e-12 * kappa`` (500x that floor).  Every other field is held to the
  pure relative tolerance (with a 1e-30 guard against exact zeros);
- the reference rounds every cell product to Float32 before its Float64 shell sum, so its
  own outputs carry rounding noise, which ill-conditioned quantities (p_v near zero, where
  l3 + l1 - 2 l2 cancels) amplify.  When the oracle's full-FP64 variant is given
  (``ora_exact``: the same walk with exact products), that noise, |ora - ora_exact|, is
  measured per peak and field and added (twice) to the tolerance: the device then has to
  agree with the reference to 1e-5 or to within the reference's own rounding noise.
"""
from __future__ import annotations

import numpy as np

SCALAR = ("RTHL", "Fbarx", "e_v", "p_v", "Srb", "d2F", "zvir_half")
VECTOR = ("Sbar", "Sbar2", "gradpk", "gradpkf", "gradpkrf", "strain", "eigs")
RATIO_FIELDS = ("e_v", "p_v")


def _as_rows(a, n):
    a = np.asarray(a, np.float64)
    return a.reshape(n, -1)


def report(gpu: dict, ora: np.ndarray, *, rel: float = 1e-5, flip_margin: float = 1e-6,
           ora_exact: np.ndarray = None, max_list: int = 20) -> dict:
    """gpu: dict of per-peak arrays (RTHL (n,), strain (n, 9) or (9 n,), ...) in the
    oracle's peak order; ora: the oracle's structured result array (oracle.RESULT_DTYPE);
    ora_exact: optionally the full-FP64 oracle's results for the same peaks.  Returns a
    JSON-ready dict: peaks, collapsed (in both), flips, flips_unexplained, mismatches,
    max_rel per field, and up to max_list listed offenders."""
    n = len(ora)
    g = {f: _as_rows(gpu[f], n) for f in SCALAR + VECTOR}
    o = {f: _as_rows(ora[f], n) for f in SCALAR + VECTOR}
    ox = {f: _as_rows(ora_exact[f], n) for f in SCALAR + VECTOR} if ora_exact is not None \
        else None
    gc = g["RTHL"][:, 0] > 0
    oc = o["RTHL"][:, 0] > 0
    flip_idx = np.flatnonzero(gc != oc)
    margins = np.asarray(ora["margin"], np.float64)[flip_idx]
    unexplained = flip_idx[~(margins < flip_margin)]
    both = gc & oc
    eig = o["eigs"]
    trace = np.abs(eig.sum(1))
    kappa = np.abs(eig).max(1) / np.where(trace > 0, trace, np.inf)
    bad = np.zeros(n, bool)
    noisy = np.zeros(n, bool)   # beyond rel, within the reference's own rounding noise
    worst_field = np.full(n, "", dtype=object)
    worst_err = np.zeros(n)
    max_rel = {}
    for f in SCALAR + VECTOR:
        gv, ov = g[f], o[f]
        nan_g, nan_o = np.isnan(gv).any(1), np.isnan(ov).any(1)
        nan_bad = both & (nan_g != nan_o)
        ok = both & ~nan_g & ~nan_o
        diff = np.abs(gv - ov).max(1)
        mag = np.abs(ov).max(1)
        err = np.zeros(n)
        noise = np.zeros(n)
        if ox is not None:
            with np.errstate(invalid="ignore"):
                noise = np.nan_to_num(np.abs(ov - ox[f]).max(1), nan=0.0)
        with np.errstate(invalid="ignore", divide="ignore"):
            err[ok] = diff[ok] / np.maximum(mag[ok], 1e-30)
            tol = rel * mag + 2.0 * noise
            if f in RATIO_FIELDS:
                tol = tol + 1e-12 * kappa
            fail = ok & (diff > tol)
            noisy |= ok & ~fail & (diff > rel * mag + (1e-12 * kappa if f in RATIO_FIELDS else 0.0))
        fail |= nan_bad
        max_rel[f] = float(err[ok].max()) if ok.any() else 0.0
        upd = fail & (err >= worst_err)
        worst_field[upd] = f
        worst_err[upd] = np.where(nan_bad[upd], np.inf, err[upd])
        bad |= fail
    mism = np.flatnonzero(bad)
    return {
        "peaks": int(n), "collapsed": int(both.sum()), "flips": int(len(flip_idx)),
        "flips_unexplained": int(len(unexplained)), "mismatches": int(len(mism)),
        "within_reference_noise": int((noisy & ~bad).sum()),
        "rel_tol": rel, "flip_margin": flip_margin, "max_rel": max_rel,
        "flip_list": [(int(p), float(ora["margin"][p])) for p in flip_idx[:max_list]],
        "mismatch_list": [(int(p), str(worst_field[p]), float(worst_err[p]))
                          for p in mism[:max_list]],
    }
