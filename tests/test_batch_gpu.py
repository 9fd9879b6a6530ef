"""Batched solver (vajra_pdhg_solve_batch): every instance to FP64 relative KKT <= 1e-6 on
its own original LP, objectives at the planted optima, per-instance fault isolation."""
import numpy as np
import pytest

import vajra_pdhg as V
from vajra_pdhg import workloads as W
from vajra_pdhg.kkt import bound_norm, relative_kkt

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


def kkt_objective_bound(lp, *sols, tol=1.05e-6):
    """How far apart the objectives of points certified at relative KKT <= tol can lie: each
    point's objective is within tol (1 + |b|) |y| + tol (1 + |c|) |x| + tol (1 + |p| + |d|) of
    the optimum (primal residual times the dual, dual residual times the primal, gap)."""
    b, c = bound_norm(lp), np.linalg.norm(lp.c)
    total = 0.0
    for r in sols:
        obj = abs(r["objective_value"])
        total += tol * ((1 + b) * np.linalg.norm(r["y"]) + (1 + c) * np.linalg.norm(r["x"]) + 1 + 2 * obj)
    return total


def test_batch_matches_single_solves(cuda):
    lps = small_batch(6, seed=6)
    res = V.solve_batch(lps)
    for lp, r in zip(lps, res):
        s = V.solve(lp, precision=V.PREC_FP64)
        for q in (r, s):
            assert relative_kkt(lp, q["x"], q["y"])["rel_kkt"] <= 1.05e-6
        assert abs(r["objective_value"] - s["objective_value"]) <= kkt_objective_bound(lp, r, s)


def test_batch_mixed_senses_and_offsets(cuda):
    lps = [W.small_random(120, 300, 31), W.small_random(80, 200, 32), W.random_planted(150, 400, 5, seed=33)]
    lps[1].sense = 1
    lps[1].c = -lps[1].c
    lps[1].objective_offset = 2.5
    res = V.solve_batch(lps)
    for lp, r in zip(lps, res):
        s = V.solve(lp, precision=V.PREC_FP64)
        assert r["status_name"] == "OPTIMAL"
        assert abs(r["objective_value"] - s["objective_value"]) <= kkt_objective_bound(lp, r, s)
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


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_iteration_limit_across_graph_launches(cuda, precision):
    """The first graph launch of a pass runs 32 chunks of 64 iterations (a WHILE node repeats
    the chunk on the device), later launches what is left up to the limit, and a last partial
    chunk runs directly.  A limit of 33 chunks + 17 iterations crosses a launch boundary and
    ends in a partial chunk.  Instances that finish
    in their first pass before it give the unlimited call's results (same status and count).  In the
    FP64-only form the others stop at exactly the limit; in mixed precision an instance's own
    count can be lower (the FP64 pass starts when the FP32 pass has ended for all)."""
    prec = V.PREC_FP64 if precision == "fp64" else V.PREC_MIXED
    lps = small_batch(8, seed=12, m_lo=3000, m_hi=8000)
    full = V.solve_batch(lps, precision=prec)
    limit = 64 * 33 + 17
    assert max(r["iterations"] for r in full) > limit, [r["iterations"] for r in full]
    lim = V.solve_batch(lps, precision=prec, iteration_limit=limit)
    for a, b in zip(full, lim):
        assert b["status_name"] in ("OPTIMAL", "ITERATION_LIMIT"), b["status_message"]
        assert b["iterations"] <= limit
        assert np.all(np.isfinite(b["x"])) and np.all(np.isfinite(b["y"]))
        if a["iterations"] <= 64 * 33 and a["fp64_iterations"] == a["iterations"] - a["fp32_iterations"] and \
                (precision == "fp64" or a["fp64_iterations"] == 0):
            # same trajectory; the set-up's timed SpMV-shape choice can differ between the two
            # calls, and with it the summation order (last-bit differences)
            assert b["status_name"] == a["status_name"] and b["iterations"] == a["iterations"]
            np.testing.assert_allclose(b["x"], a["x"], rtol=1e-8, atol=1e-8)
            np.testing.assert_allclose(b["y"], a["y"], rtol=1e-8, atol=1e-8)
        elif precision == "fp64" and a["iterations"] > limit:
            assert b["status_name"] == "ITERATION_LIMIT", b["status_message"]
            assert b["iterations"] == limit
    if precision == "fp64":
        assert sum(r["status_name"] == "ITERATION_LIMIT" for r in lim) >= 1


def rows_scaled(lp, seed, decades=3.0):
    """The same LP with row i of A and of its bounds multiplied by 10^u, u ~ U[-decades, decades]
    (same sparsity, same solution x; Ruiz needs several more passes to balance it)."""
    rng = np.random.default_rng(seed)
    d = 10.0 ** rng.uniform(-decades, decades, size=lp.num_rows)
    q = W.LP(**{**lp.__dict__})
    q.values = lp.values * d[lp.row_idx]
    q.row_lower = np.where(lp.row_lower > -1e20, lp.row_lower * d, lp.row_lower)
    q.row_upper = np.where(lp.row_upper < 1e20, lp.row_upper * d, lp.row_upper)
    q.y_planted = None
    return q


def test_batch_scales_each_instance_as_alone(cuda):
    """Each instance ends its Ruiz passes on its own stopping test.  Instance A is solved next to
    B and next to C, where C is B with its rows scaled over six decades (same sparsity, so the
    set-up picks the same SpMV shapes with autotuning off; C needs many more Ruiz passes than
    B).  A's results must be bit-identical in both batches; with one stopping test over the
    packed matrix, A would take C's extra passes in the second batch."""
    a = W.random_planted(300, 800, 6, seed=71)
    b = W.random_planted(400, 1000, 6, seed=72)
    c = rows_scaled(b, seed=73)
    kw = dict(precision=V.PREC_FP64, autotune=0, iteration_limit=20000)
    with_b = V.solve_batch([a, b], **kw)
    with_c = V.solve_batch([a, c], **kw)
    assert with_b[0]["status_name"] == "OPTIMAL"
    assert with_b[0]["iterations"] == with_c[0]["iterations"]
    np.testing.assert_array_equal(with_b[0]["x"], with_c[0]["x"])
    np.testing.assert_array_equal(with_b[0]["y"], with_c[0]["y"])
    assert with_b[0]["spectral_norm_estimate"] == with_c[0]["spectral_norm_estimate"]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_time_limit(cuda, precision):
    """The time limit is checked after every launch of a pass graph (the first one runs 32
    chunks of 64 iterations, later ones what fits in the time left): with 1 ms, the call ends
    after its first launch; instances not finished by then report TIME_LIMIT with finite
    points (in mixed precision, their FP32 candidates)."""
    prec = V.PREC_FP64 if precision == "fp64" else V.PREC_MIXED
    lps = small_batch(8, seed=12, m_lo=3000, m_hi=8000)
    res = V.solve_batch(lps, precision=prec, time_limit=1e-3)
    names = [r["status_name"] for r in res]
    assert "TIME_LIMIT" in names, names
    for r in res:
        assert r["status_name"] in ("OPTIMAL", "TIME_LIMIT"), r["status_message"]
        assert r["iterations"] <= 32 * 64
        assert np.all(np.isfinite(r["x"])) and np.all(np.isfinite(r["y"]))
