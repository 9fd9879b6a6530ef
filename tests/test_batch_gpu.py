"""Batched solver (vajra_pdhg_solve_batch): every instance to FP64 relative KKT <= 1e-6 on
its own original LP, objectives at the planted optima, per-instance fault isolation."""
import numpy as np
import pytest

import vajra_pdhg as V
from vajra_pdhg import workloads as W
from vajra_pdhg.kkt import relative_kkt

pytestmark = pytest.mark.gpu


def small_batch(count, seed, m_lo=60, m_hi=1500):
    sizes = W.batch_sizes(count, seed=seed, m_lo=m_lo, m_hi=m_hi)
    return [W.random_planted(m, n, k, seed=seed * 1000 + i) for i, (m, n, k) in enumerate(sizes)]


def test_batch_reaches_planted_optima(cuda):
    lps = small_batch(24, seed=5)
    res = V.solve_batch(lps)
    for lp, r in zip(lps, res):
        assert r["status_name"] == "OPTIMAL", r["status_message"]
        k = relative_kkt(lp, r["x"], r["y"])
        assert r["rel_kkt"] <= 1e-6 and k["rel_kkt"] <= 1.05e-6, (r["rel_kkt"], k)
        rel = abs(r["objective_value"] - lp.planted_objective) / (1 + abs(lp.planted_objective))
        assert rel <= 1e-5, rel
        np.testing.assert_allclose(r["row_value"], lp.to_scipy_csc() @ r["x"], rtol=1e-12, atol=1e-9)


def test_batch_matches_single_solves(cuda):
    lps = small_batch(6, seed=6)
    res = V.solve_batch(lps)
    for lp, r in zip(lps, res):
        s = V.solve(lp, precision=V.PREC_FP64)
        assert abs(r["objective_value"] - s["objective_value"]) <= 1e-5 * (1 + abs(s["objective_value"]))


def test_batch_mixed_senses_and_offsets(cuda):
    lps = [W.small_random(120, 300, 31), W.small_random(80, 200, 32), W.random_planted(150, 400, 5, seed=33)]
    lps[1].sense = 1
    lps[1].c = -lps[1].c
    lps[1].objective_offset = 2.5
    res = V.solve_batch(lps)
    for lp, r in zip(lps, res):
        s = V.solve(lp, precision=V.PREC_FP64)
        assert r["status_name"] == "OPTIMAL"
        assert abs(r["objective_value"] - s["objective_value"]) <= 1e-5 * (1 + abs(s["objective_value"]))
        assert relative_kkt(lp, r["x"], r["y"])["rel_kkt"] <= 1.05e-6


def test_batch_isolates_a_failing_instance(cuda):
    lps = small_batch(5, seed=7)
    lps[2].c = lps[2].c.copy()
    lps[2].c[0] = np.nan
    res = V.solve_batch(lps)
    assert res[2]["status_name"] == "NUMERICAL_ERROR"
    for i in (0, 1, 3, 4):
        assert res[i]["status_name"] == "OPTIMAL"


def test_batch_iteration_limit(cuda):
    lps = small_batch(4, seed=8)
    res = V.solve_batch(lps, iteration_limit=64)
    for r in res:
        assert r["status_name"] in ("ITERATION_LIMIT", "OPTIMAL")
        assert r["iterations"] <= 64


def test_batch_mixed_and_fp64_passes(cuda):
    """Mixed precision: every instance runs an FP32 pass first and finishes there or in the FP64
    pass after its hand-over; the plain form runs FP64 only.  Both reach the planted optima."""
    lps = small_batch(12, seed=9)
    mixed = V.solve_batch(lps, precision=V.PREC_MIXED)
    plain = V.solve_batch(lps, precision=V.PREC_FP64)
    assert any(r["fp32_iterations"] > 0 for r in mixed)
    assert all(r["fp32_iterations"] == 0 for r in plain)
    for lp, a, b in zip(lps, mixed, plain):
        for r in (a, b):
            assert r["status_name"] == "OPTIMAL", r["status_message"]
            assert r["fp32_iterations"] + r["fp64_iterations"] == r["iterations"]
            assert relative_kkt(lp, r["x"], r["y"])["rel_kkt"] <= 1.05e-6
            assert abs(r["objective_value"] - lp.planted_objective) <= 1e-5 * (1 + abs(lp.planted_objective))


def test_batch_mixed_iteration_limit_inside_the_fp32_pass(cuda):
    """A limit reached in the FP32 pass reports the FP32 candidates, widened, as limit results."""
    lps = small_batch(4, seed=10)
    res = V.solve_batch(lps, precision=V.PREC_MIXED, iteration_limit=128)
    for lp, r in zip(lps, res):
        assert r["status_name"] in ("ITERATION_LIMIT", "OPTIMAL")
        assert r["iterations"] <= 128 and r["fp64_iterations"] == 0
        assert np.all(np.isfinite(r["x"])) and np.all(np.isfinite(r["y"]))
