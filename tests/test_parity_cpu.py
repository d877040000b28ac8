"""oracle/parity.py, the report the GPU parity tests and the benchmark use, checked on the
CPU with mistakes planted in copies of oracle results (no device involved)."""
import numpy as np

from oracle import RESULT_DTYPE, parity


def _oracle_rows(n, rng):
    o = np.zeros(n, dtype=RESULT_DTYPE)
    for name in RESULT_DTYPE.names:
        o[name] = rng.uniform(0.5, 2.0, o[name].shape)
    o["eigs"] = np.sort(rng.uniform(0.2, 1.0, (n, 3)), axis=1)
    o["margin"] = 1.0
    return o


def _as_gpu(o):
    return {f: np.array(o[f], np.float64).reshape(len(o), -1) for f in parity.SCALAR + parity.VECTOR}


def test_identical_results_pass():
    o = _oracle_rows(50, np.random.default_rng(0))
    rep = parity.report(_as_gpu(o), o)
    assert rep["mismatches"] == 0 and rep["flips"] == 0 and rep["collapsed"] == 50


def test_relative_error_above_tolerance_is_a_mismatch():
    o = _oracle_rows(50, np.random.default_rng(1))
    g = _as_gpu(o)
    g["Srb"][7, 0] *= 1 + 3e-5
    g["gradpk"][9, 1] *= 1 + 5e-6          # within 1e-5: accepted
    rep = parity.report(g, o)
    assert rep["mismatches"] == 1 and rep["mismatch_list"][0][:2] == (7, "Srb")


def test_flip_needs_a_small_decision_margin():
    o = _oracle_rows(20, np.random.default_rng(2))
    o["RTHL"][3] = -1.0                    # the oracle says: no collapse
    o["margin"][3] = 4e-7                  # decided within round-off of the barrier
    o["RTHL"][5] = -1.0
    o["margin"][5] = 0.3                   # decided far from the barrier
    g = _as_gpu(o)
    g["RTHL"][3, 0] = 2.0
    g["RTHL"][5, 0] = 2.0
    rep = parity.report(g, o)
    assert rep["flips"] == 2 and rep["flips_unexplained"] == 1
    assert [p for p, _ in rep["flip_list"]] == [3, 5]


def test_ratio_fields_get_the_cancellation_floor():
    o = _oracle_rows(4, np.random.default_rng(3))
    # an ill-conditioned trace: eigenvalues 1e3 apart around a trace of 1e-2
    o["eigs"][0] = (-500.0, 0.005, 500.005)
    o["p_v"][0] = 1e-9
    g = _as_gpu(o)
    g["p_v"][0, 0] = 1e-9 + 1e-8          # 1e-8 absolute: below 1e-12 kappa (kappa ~ 5e4)
    rep = parity.report(g, o)
    assert rep["mismatches"] == 0
    g["p_v"][0, 0] = 1e-9 + 1e-6          # far above the floor
    assert parity.report(g, o)["mismatches"] == 1


def test_nan_on_one_side_only_is_a_mismatch():
    o = _oracle_rows(5, np.random.default_rng(4))
    o["zvir_half"][2] = np.nan
    g = _as_gpu(o)
    assert parity.report(g, o)["mismatches"] == 0
    g["zvir_half"][2, 0] = 1.0
    assert parity.report(g, o)["mismatches"] == 1


def test_reference_rounding_noise_widens_the_tolerance():
    o = _oracle_rows(6, np.random.default_rng(5))
    ox = o.copy()
    ox["p_v"][1] *= 1 + 4e-4          # the reference's own products move p_v by 4e-4 here
    g = _as_gpu(ox)                    # the device agrees with the exact-product oracle
    rep = parity.report(g, o)
    assert rep["mismatches"] == 1
    rep = parity.report(g, o, ora_exact=ox)
    assert rep["mismatches"] == 0 and rep["within_reference_noise"] == 1
    g["p_v"][1, 0] = o["p_v"][1] * (1 + 2e-3)   # beyond twice the noise: still a mismatch
    assert parity.report(g, o, ora_exact=ox)["mismatches"] == 1
