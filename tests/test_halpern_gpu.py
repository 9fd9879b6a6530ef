"""VAJRA_ALGO_HALPERN (restarted reflected Halpern PDHG) on the device, FP64 and mixed:
relative KKT <= 1e-6 verified independently in FP64 on the host, objective against the
planted optimum / HiGHS, the reference's own KKT verifier, determinism and limits."""
import numpy as np
import pytest
import scipy.optimize as so

import vajra_pdhg as V
from oracle import bindings as B
from vajra_pdhg import workloads as W
from vajra_pdhg.kkt import bound_norm, relative_kkt

pytestmark = pytest.mark.gpu
INF = 1e20
PRECISIONS = [V.PREC_FP64, V.PREC_MIXED]


def highs(lp):
    A = lp.to_scipy_csc()
    sign = -1.0 if lp.sense else 1.0
    rl, ru = lp.row_lower, lp.row_upper
    eq = (rl == ru)
    A_ub, b_ub = [], []
    import scipy.sparse as sp
    up = (~eq) & (ru < INF)
    lo = (~eq) & (rl > -INF)
    A_ub = sp.vstack([A[up], -A[lo]]) if (up.any() or lo.any()) else None
    b_ub = np.concatenate([ru[up], -rl[lo]]) if A_ub is not None else None
    bounds = list(zip(np.where(lp.col_lower > -INF, lp.col_lower, None), np.where(lp.col_upper < INF, lp.col_upper, None)))
    res = so.linprog(sign * lp.c, A_ub=A_ub, b_ub=b_ub, A_eq=A[eq] if eq.any() else None,
                     b_eq=rl[eq] if eq.any() else None, bounds=bounds, method="highs")
    assert res.status == 0, res.message
    return sign * res.fun + lp.objective_offset


def check_solution(lp, g, tol=1e-6, obj=None, obj_tol=1e-5):
    assert g["status_name"] == "OPTIMAL", g["status_message"]
    assert g["rel_kkt"] <= tol
    k = relative_kkt(lp, g["x"], g["y"])
    assert k["rel_kkt"] <= 1.05 * tol + 1e-12, k            # host FP64 check of the device figure
    assert abs(k["rel_kkt"] - g["rel_kkt"]) <= 1e-8 + 1e-3 * g["rel_kkt"], (k, g["rel_kkt"])
    assert abs(g["objective_value"] - k["primal_objective"] * (-1 if lp.sense else 1)) <= 1e-7 * (1 + abs(g["objective_value"]))
    if obj is not None:
        assert abs(g["objective_value"] - obj) <= obj_tol * (1 + abs(obj)), (g["objective_value"], obj)
    np.testing.assert_allclose(g["row_value"], lp.to_scipy_csc() @ g["x"], rtol=1e-12, atol=1e-9)
    if B.ref_available():
        # The reference verifier (absolute tolerances) at the violation size a relative KKT
        # of `tol` allows: tol (1 + ||b||) for rows, tol (1 + ||c||) for reduced costs.
        vt = max(1e-9, tol * (1.0 + max(bound_norm(lp), np.linalg.norm(lp.c))))
        v = B.ref_verify(lp, g["x"], g["y"], g["objective_value"], g["status"], tol=vt)
        assert v["passed"], v["summary"]


@pytest.mark.parametrize("prec", PRECISIONS)
@pytest.mark.parametrize("m,n,seed", [(200, 500, 0), (2000, 5000, 1)])
def test_planted_optimum(cuda, prec, m, n, seed):
    lp = W.random_planted(m, n, 8, seed=seed)
    g = V.solve(lp, precision=prec)
    check_solution(lp, g, obj=lp.planted_objective)
    if B.ref_available():
        # The reference verifier checks absolute violations; a relative KKT of 1e-6 bounds
        # every single violation by 1e-6 (1 + ||b||) (primal) and 1e-6 (1 + ||c||) (dual).
        tol = 1e-6 * (1.0 + max(bound_norm(lp), np.linalg.norm(lp.c)))
        v = B.ref_verify(lp, g["x"], g["y"], g["objective_value"], g["status"], tol=tol)
        assert v["passed"], v["summary"]


@pytest.mark.parametrize("prec", PRECISIONS)
@pytest.mark.parametrize("seed", [3, 4])
def test_mixed_senses_vs_highs(cuda, prec, seed):
    lp = W.small_random(300, 700, seed)
    g = V.solve(lp, precision=prec)
    check_solution(lp, g, obj=highs(lp))


@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("prec", PRECISIONS)
def test_maximise_free_columns_vs_highs(cuda, prec, order):
    lp = W.small_random(150, 400, 9)
    lp.sense = 1
    lp.c = -lp.c
    lp.objective_offset = 3.5
    lp.col_lower = lp.col_lower.copy(); lp.col_upper = lp.col_upper.copy()
    lp.col_lower[::11] = -INF
    g = V.solve(lp, precision=prec, degree_order=order)
    check_solution(lp, g, obj=highs(lp))


@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("prec", PRECISIONS)
def test_min_cost_flow_vs_highs(cuda, prec, order):
    lp = W.min_cost_flow(nodes=2000, arcs=15000, seed=5)
    g = V.solve(lp, precision=prec, degree_order=order)
    check_solution(lp, g, obj=highs(lp))


PDHG_TEST_OPTIMA = [   # tests/test_pdhg.cpp LPs and optima
    ((3, 2, [(0, 0, 1), (0, 1, 1), (1, 0, 1), (2, 1, 1)], [-1, -2], [0, 0], [INF, INF], [-INF] * 3, [4, 3, 3], 0), -7.0),
    ((2, 3, [(0, 0, 1), (0, 1, 1), (0, 2, 1), (1, 0, 2), (1, 1, 1)], [1, 2, 3], [0] * 3, [INF] * 3, [6, 5], [6, 5], 0), 13.0),
    ((3, 2, [(0, 0, 1), (0, 1, 1), (1, 0, 1), (1, 1, -1), (2, 0, 2), (2, 1, 1)], [2, 3], [0, 0], [10, 10],
      [2, -INF, 1], [INF, 4, 6], 0), 4.0),
    ((1, 2, [(0, 0, 1), (0, 1, 1)], [2, 1], [-10, -INF], [10, INF], [5], [5], 0), -5.0),
    ((1, 2, [(0, 0, 1), (0, 1, 1)], [-2, -3], [0, 0], [INF, INF], [-INF], [5], 0), -15.0),
    ((1, 2, [(0, 0, 1), (0, 1, 1)], [2, 3], [0, 0], [INF, INF], [-INF], [5], 1), 15.0),
    ((1, 2, [(0, 0, 1), (0, 1, 1)], [1, 1], [0, 0], [10, 10], [3], [10], 0), 3.0),
]


@pytest.mark.parametrize("prec", PRECISIONS)
@pytest.mark.parametrize("case", range(len(PDHG_TEST_OPTIMA)))
def test_reference_test_lps_reach_optimum(cuda, prec, case):
    (m, n, trips, c, cl, cu, rl, ru, sense), opt = PDHG_TEST_OPTIMA[case]
    cp, ri, vals = W.canonical_csc(m, n, [t[0] for t in trips], [t[1] for t in trips], [t[2] for t in trips])
    lp = W.LP(m, n, cp, ri, vals, np.array(c, float), np.array(cl, float), np.array(cu, float), np.array(rl, float),
              np.array(ru, float), sense=sense)
    g = V.solve(lp, precision=prec)
    check_solution(lp, g, obj=opt)


@pytest.mark.parametrize("shape", [-1, -2, 1, 2, 4, 8, 16, 32])
@pytest.mark.parametrize("prec", PRECISIONS)
def test_every_spmv_shape_reaches_the_optimum(cuda, prec, shape):
    """Each launch shape of the iteration kernels (row blocks with one or two load groups,
    1..32 lanes per row), forced for both SpMVs, solves to the tolerance."""
    lp = W.random_planted(600, 1500, (2, 40), seed=31)
    g = V.solve(lp, precision=prec, spmv_shape_a=shape, spmv_shape_at=shape)
    want = 0 if shape == -1 else (64 if shape == -2 else shape)
    assert g["spmv_group_a"] == want and g["spmv_group_at"] == want
    check_solution(lp, g, obj=lp.planted_objective)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_deterministic(cuda, prec):
    lp = W.random_planted(500, 1200, 6, seed=21)
    with V.Solver(lp, precision=prec) as s:
        a, b = s.run(), s.run()
    for k in ("x", "y", "d", "row_value"):
        np.testing.assert_array_equal(a[k], b[k])
    assert a["iterations"] == b["iterations"] and a["rel_kkt"] == b["rel_kkt"]


def test_iteration_limit_and_partial_chunk(cuda):
    lp = W.random_planted(500, 1200, 6, seed=22)
    g = V.solve(lp, precision=V.PREC_FP64, iteration_limit=100)
    assert g["status_name"] == "ITERATION_LIMIT" and g["iterations"] == 100
    g = V.solve(lp, precision=V.PREC_FP64, iteration_limit=0)
    assert g["status_name"] == "ITERATION_LIMIT" and g["iterations"] == 0


def test_nan_objective_is_numerical_error(cuda):
    lp = W.random_planted(100, 250, 5, seed=23)
    lp.c = lp.c.copy(); lp.c[3] = np.nan
    g = V.solve(lp, precision=V.PREC_FP64)
    assert g["status_name"] == "NUMERICAL_ERROR"


def test_mixed_splits_iterations(cuda):
    lp = W.random_planted(2000, 5000, 8, seed=24)
    g = V.solve(lp, precision=V.PREC_MIXED)
    assert g["fp32_iterations"] > 0 and g["fp32_iterations"] + g["fp64_iterations"] == g["iterations"]


def with_structure(lp, dense_row=None, dense_col=None, empty_rows=(), empty_cols=(), seed=0):
    """lp with one dense row / column added to A and some rows / columns emptied (their bounds
    kept satisfiable), rebuilt through the canonical CSC of the generators."""
    rng = np.random.default_rng(seed)
    A = lp.to_scipy_csc().tocoo()
    keep = ~np.isin(A.row, list(empty_rows)) & ~np.isin(A.col, list(empty_cols))
    r, c, v = list(A.row[keep]), list(A.col[keep]), list(A.data[keep])
    if dense_row is not None:
        cols = np.setdiff1d(np.arange(lp.num_cols), list(empty_cols))
        r += [dense_row] * len(cols); c += list(cols); v += list(rng.uniform(-1e-3, 1e-3, len(cols)))
    if dense_col is not None:
        rows = np.setdiff1d(np.arange(lp.num_rows), list(empty_rows))
        r += list(rows); c += [dense_col] * len(rows); v += list(rng.uniform(-1e-3, 1e-3, len(rows)))
    cp, ri, vals = W.canonical_csc(lp.num_rows, lp.num_cols, np.array(r), np.array(c), np.array(v))
    out = W.LP(lp.num_rows, lp.num_cols, cp, ri, vals, lp.c.copy(), lp.col_lower.copy(), lp.col_upper.copy(),
               lp.row_lower.copy(), lp.row_upper.copy(), sense=lp.sense)
    x = np.clip(np.zeros(lp.num_cols), out.col_lower, out.col_upper)
    ax = out.to_scipy_csc() @ x
    # feasible by construction: every row range holds A x0 for the bound-clipped x0 = 0 point
    out.row_lower = np.where(out.row_lower > -INF, np.minimum(out.row_lower, ax - 1.0), out.row_lower)
    out.row_upper = np.where(out.row_upper < INF, np.maximum(out.row_upper, ax + 1.0), out.row_upper)
    for i in empty_rows:
        out.row_lower[i], out.row_upper[i] = -1.0, 1.0
    return out


@pytest.mark.parametrize("shape", [-1, -2, 4, 32])
def test_long_rows_and_empty_rows_and_columns(cuda, shape):
    """A row and a column longer than a row block (2048 entries: the one-CTA-per-row paths of
    both kernels) plus empty rows and columns, under the fixed launch shapes."""
    base = W.small_random(2600, 3000, 12)
    lp = with_structure(base, dense_row=7, dense_col=11, empty_rows=(3, 50, 2599), empty_cols=(0, 99, 2999), seed=1)
    nnz = np.diff(lp.col_ptr)
    assert nnz.max() > 2048 and (nnz == 0).sum() >= 3
    g = V.solve(lp, precision=V.PREC_FP64, spmv_shape_a=shape, spmv_shape_at=shape)
    check_solution(lp, g, obj=highs(lp))


@pytest.mark.parametrize("prec", PRECISIONS)
def test_infeasible_lp_is_not_reported_optimal(cuda, prec):
    # x0 + x1 >= 4 and x0 + x1 <= 1 with 0 <= x <= 10
    cp, ri, vals = W.canonical_csc(2, 2, np.array([0, 0, 1, 1]), np.array([0, 1, 0, 1]), np.ones(4))
    lp = W.LP(2, 2, cp, ri, vals, np.array([1.0, 1.0]), np.zeros(2), np.full(2, 10.0), np.array([4.0, -INF]),
              np.array([INF, 1.0]))
    g = V.solve(lp, precision=prec, iteration_limit=20000)
    assert g["status_name"] != "OPTIMAL"
    assert g["rel_kkt"] > 1e-6


def test_time_limit_stops_the_solve(cuda):
    lp = W.random_planted(2000, 5000, 8, seed=5)
    g = V.solve(lp, precision=V.PREC_FP64, time_limit=1e-4)
    assert g["status_name"] == "TIME_LIMIT"
    assert g["iterations"] < 5000


@pytest.mark.parametrize("prec", PRECISIONS)
def test_degree_order_reaches_the_optimum(cuda, prec):
    """Rows and columns renumbered by entry count on the device (forced on for a small LP with
    2..40 entries a column): the solution comes back in the caller's numbering and passes every
    check of the unordered solve."""
    lp = W.random_planted(600, 1500, (2, 40), seed=31)
    g = V.solve(lp, precision=prec, degree_order=1)
    check_solution(lp, g, obj=lp.planted_objective)


def test_degree_order_with_long_and_empty_rows_and_columns(cuda):
    """The ordering with a row and a column longer than a row block and empty rows and columns.
    FP64: on this LP the mixed solution (relative KKT 2.8e-7, ordered or not) leaves one
    reduced cost 2 % above the reference verifier's absolute dual tolerance."""
    base = W.small_random(2600, 3000, 12)
    lp = with_structure(base, dense_row=7, dense_col=11, empty_rows=(3, 50, 2599), empty_cols=(0, 99, 2999), seed=1)
    g = V.solve(lp, precision=V.PREC_FP64, degree_order=1)
    check_solution(lp, g, obj=highs(lp))


def test_degree_order_returns_the_callers_numbering(cuda):
    """64 FP64 iterations with and without the ordering: the ordering changes summation orders
    only, so the iterates agree to rounding; a wrong renumbering would differ at O(1)."""
    lp = W.random_planted(1500, 4000, (2, 40), seed=33)
    kw = dict(precision=V.PREC_FP64, iteration_limit=64, spmv_shape_a=-1, spmv_shape_at=-1)
    a = V.solve(lp, degree_order=1, **kw)
    b = V.solve(lp, degree_order=-1, **kw)
    assert a["iterations"] == b["iterations"] == 64
    for k in ("x", "y", "d", "row_value"):
        np.testing.assert_allclose(a[k], b[k], rtol=1e-7, atol=1e-9 * (1.0 + np.abs(b[k]).max()), err_msg=k)
    assert abs(a["objective_value"] - b["objective_value"]) <= 1e-9 * (1.0 + abs(b["objective_value"]))


@pytest.mark.parametrize("prec", PRECISIONS)
def test_sliced_ell_shape_reaches_the_optimum(cuda, prec):
    """The sliced-ELL kernels (shape -3, built only for degree-ordered LPs), forced for both
    SpMVs: rows of 2..40 entries in slices of 32, reported as group 128."""
    lp = W.random_planted(600, 1500, (2, 40), seed=31)
    g = V.solve(lp, precision=prec, degree_order=1, spmv_shape_a=-3, spmv_shape_at=-3)
    assert g["spmv_group_a"] == 128 and g["spmv_group_at"] == 128
    check_solution(lp, g, obj=lp.planted_objective)


def test_sliced_ell_long_rows_and_empty_rows_and_columns(cuda):
    """Sliced ELL with a row of ~5000 entries (one CTA), a column of ~2600 (one warp), rows
    above 128 entries kept in CSR, and empty rows and columns."""
    base = W.small_random(2600, 5000, 12)
    lp = with_structure(base, dense_row=7, dense_col=11, empty_rows=(3, 50, 2599), empty_cols=(0, 99, 4999), seed=1)
    A = lp.to_scipy_csc()
    assert np.diff(A.tocsr().indptr).max() > 4096 and np.diff(lp.col_ptr).max() > 128
    g = V.solve(lp, precision=V.PREC_FP64, degree_order=1, spmv_shape_a=-3, spmv_shape_at=-3)
    assert g["spmv_group_a"] == 128 and g["spmv_group_at"] == 128
    check_solution(lp, g, obj=highs(lp))


def test_sliced_ell_matches_row_blocks(cuda):
    """64 FP64 iterations in sliced ELL and in row blocks: only the summation order differs,
    so the iterates agree to rounding; a misplaced entry would differ at O(1)."""
    lp = W.random_planted(900, 4000, (2, 50), seed=34)   # rows on both sides of 128 entries: slices and warps
    kw = dict(precision=V.PREC_FP64, iteration_limit=64, degree_order=1)
    a = V.solve(lp, spmv_shape_a=-3, spmv_shape_at=-3, **kw)
    b = V.solve(lp, spmv_shape_a=-1, spmv_shape_at=-1, **kw)
    assert a["spmv_group_a"] == 128 and b["spmv_group_a"] == 0
    for k in ("x", "y", "d", "row_value"):
        np.testing.assert_allclose(a[k], b[k], rtol=1e-7, atol=1e-9 * (1.0 + np.abs(b[k]).max()), err_msg=k)


def test_sliced_ell_shape_without_ordering(cuda):
    """Without the degree ordering a forced shape -3 builds the sliced copy over rows in their
    own order (slices of uneven rows, long rows listed wherever they are) and solves the same."""
    base = W.small_random(2600, 5000, 12)
    lp = with_structure(base, dense_row=7, dense_col=11, empty_rows=(3, 50, 2599), empty_cols=(0, 99, 4999), seed=1)
    g = V.solve(lp, precision=V.PREC_FP64, degree_order=-1, spmv_shape_a=-3, spmv_shape_at=-3)
    assert g["spmv_group_a"] == 128 and g["spmv_group_at"] == 128
    check_solution(lp, g, obj=highs(lp))


@pytest.mark.parametrize("prec", PRECISIONS)
def test_sliced_ell_hot_prefix_shape_reaches_the_optimum(cuda, prec):
    """The sliced-ELL kernels that serve the first vector entries from shared memory (shape
    -4, reported as 129), forced for both SpMVs."""
    lp = W.random_planted(600, 1500, (2, 40), seed=31)
    g = V.solve(lp, precision=prec, degree_order=1, spmv_shape_a=-4, spmv_shape_at=-4)
    assert g["spmv_group_a"] == 129 and g["spmv_group_at"] == 129
    check_solution(lp, g, obj=lp.planted_objective)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_sliced_ell_hot_prefix_is_bit_identical_to_sliced_ell(cuda, prec):
    """Same row sums in the same order, only the source of the gathered entries differs: 64
    iterations with shape -4 and with shape -3 give the same bits.  The LP has a row above 4096
    entries (one CTA), columns of 128..4096 entries (one warp) and more columns than the hot
    prefix holds in FP64 (14,336) and in FP32 (28,672)."""
    base = W.small_random(2600, 40000, 12)
    lp = with_structure(base, dense_row=7, dense_col=11, empty_rows=(3, 50), empty_cols=(0, 99), seed=1)
    kw = dict(precision=prec, iteration_limit=64, degree_order=1)
    a = V.solve(lp, spmv_shape_a=-4, spmv_shape_at=-4, **kw)
    b = V.solve(lp, spmv_shape_a=-3, spmv_shape_at=-3, **kw)
    assert a["spmv_group_a"] == 129 and b["spmv_group_a"] == 128
    for k in ("x", "y", "d", "row_value"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def fp32_exact(lp):
    """lp with its matrix values rounded to FP32 (every value then fits FP32 exactly)."""
    out = W.LP(**{**lp.__dict__})
    out.values = np.asarray(lp.values, np.float32).astype(np.float64)
    return out


@pytest.mark.parametrize("prec", PRECISIONS)
def test_power_of_two_scaling_reaches_the_optimum(cuda, prec):
    lp = W.small_random(300, 700, 3)
    g = V.solve(lp, precision=prec, pow2_scaling=1)
    check_solution(lp, g, obj=highs(lp))


@pytest.mark.parametrize("shape", [-1, -3, -4])
def test_fp64_iterations_on_the_exact_fp32_copy_are_bit_identical(cuda, shape):
    """With power-of-two scaling an LP whose values fit FP32 keeps fitting FP32 once scaled; the
    FP64 iterations and checks may then read the FP32 copy of the matrix (FP64 vectors and
    sums): 256 iterations give the same bits as with the FP64 copy."""
    lp = fp32_exact(W.random_planted(900, 4000, (2, 50), seed=34))
    kw = dict(precision=V.PREC_FP64, iteration_limit=256, degree_order=1, pow2_scaling=1, spmv_shape_a=shape,
              spmv_shape_at=shape)
    a = V.solve(lp, fp64_value_storage=2, **kw)
    b = V.solve(lp, fp64_value_storage=1, **kw)
    assert a["primal_kernel_bytes"] < b["primal_kernel_bytes"]      # the 4-byte copy was read
    for k in ("x", "y", "d", "row_value"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert a["rel_kkt"] == b["rel_kkt"]


def test_mixed_polish_on_the_exact_fp32_copy_reaches_the_optimum(cuda):
    lp = fp32_exact(W.random_planted(2000, 5000, 8, seed=1))
    g = V.solve(lp, precision=V.PREC_MIXED, pow2_scaling=1, degree_order=1)
    check_solution(lp, g, obj=lp.planted_objective)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_max_violation_criterion_meets_the_status_guard(cuda, prec):
    """max_violation / max_abs_violation: OPTIMAL only once the status guard's maxima (row
    violation over 1 + |bound|, reduced-cost and row-dual sign violations) and the absolute row
    violations are below them, checked on the host; the reported residuals are those maxima."""
    from vajra_pdhg.kkt import guard_maxima
    lp = W.small_random(300, 700, 4)
    g = V.solve(lp, precision=prec, max_violation=5e-8, max_abs_violation=5e-7, iteration_limit=200000)
    assert g["status_name"] == "OPTIMAL" and g["rel_kkt"] <= 1e-6, (g["status_name"], g["primal_residual"],
                                                                    g["dual_residual"], g["rel_kkt"])
    q = guard_maxima(lp, g["x"], g["y"])
    assert q["primal_rel"] <= 5.05e-8 and q["dual_abs"] <= 5.05e-8 and q["primal_abs"] <= 5.05e-7, q
    assert abs(g["primal_residual"] - q["primal_abs"]) <= 1e-9 + 1e-6 * q["primal_abs"]
    plain = V.solve(lp, precision=prec)
    assert g["iterations"] >= plain["iterations"]


def test_release_cached_memory_returns_blocks_to_the_driver(cuda):
    import torch
    lp = W.random_planted(2000, 5000, 8, seed=1)
    V.solve(lp, precision=V.PREC_MIXED)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    freed = V.release_cached_memory(0)
    assert freed > 0
    assert torch.cuda.mem_get_info()[0] >= free0 + freed // 2
    assert V.release_cached_memory(0) == 0


def test_concurrent_solves_reuse_blocks_safely(cuda):
    """Solves on two host threads (two handles, two streams) share the block cache: a block one
    solve releases is handed to the other only after the releasing stream's queued work is
    done.  Every result equals the same solve run alone (solves are deterministic)."""
    import threading
    lps = [W.random_planted(1500, 4000, 6, seed=s) for s in (41, 42)]
    alone = [V.solve(lp, precision=V.PREC_FP64) for lp in lps]
    out = [[None, None] for _ in lps]

    def worker(k):
        for rep in range(2):
            out[k][rep] = V.solve(lps[k], precision=V.PREC_FP64)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for k in range(2):
        for rep in range(2):
            for key in ("x", "y", "d"):
                np.testing.assert_array_equal(out[k][rep][key], alone[k][key], err_msg=f"{k} {rep} {key}")


def test_mixed_handover_continuing_the_fp32_epoch_reaches_the_optimum(cuda):
    """handover_mode = 1: the FP64 phase takes over the FP32 phase's iterate, anchor, Halpern
    counter and restart references instead of restarting from the FP32 candidate."""
    lp = W.random_planted(2000, 5000, 8, seed=24)
    g = V.solve(lp, precision=V.PREC_MIXED, handover_mode=1, mixed_switch_tolerance=1e-4)
    assert g["fp32_iterations"] > 0 and g["fp64_iterations"] > 0
    check_solution(lp, g, obj=lp.planted_objective)


def test_chained_launch_changes_no_result(cuda, tmp_path):
    """The SpMV kernels run under programmatic dependent launch by default (each waits for the
    previous kernel's completion before its first access); VAJRA_PDL=0 launches them plainly.
    Same LP, same launch shapes (the set-up heuristic below 2^20 entries): bit-identical
    iterates, iteration counts and statuses in both precisions."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = tmp_path / "plain.npz"
    script = (
        "import sys, numpy as np\n"
        "import vajra_pdhg as V\n"
        "from vajra_pdhg import workloads as W\n"
        "lp = W.random_planted(2000, 5000, 8, seed=0)\n"
        "res = {}\n"
        "for name, p in (('fp64', V.PREC_FP64), ('mixed', V.PREC_MIXED)):\n"
        "    r = V.solve(lp, precision=p)\n"
        "    res[name + '_x'] = r['x']; res[name + '_y'] = r['y']\n"
        "    res[name + '_it'] = np.array([r['iterations'], r['status']])\n"
        f"np.savez({str(out)!r}, **res)\n")
    env = dict(os.environ, VAJRA_PDL="0",
               PYTHONPATH=os.pathsep.join([root, os.path.join(root, "vajra-opt_b200"), os.environ.get("PYTHONPATH", "")]))
    subprocess.run([sys.executable, "-c", script], env=env, check=True, timeout=600)
    plain = np.load(out)
    lp = W.random_planted(2000, 5000, 8, seed=0)
    for name, p in (("fp64", V.PREC_FP64), ("mixed", V.PREC_MIXED)):
        r = V.solve(lp, precision=p)
        assert r["status_name"] == "OPTIMAL"
        assert [r["iterations"], r["status"]] == plain[name + "_it"].tolist()
        np.testing.assert_array_equal(r["x"], plain[name + "_x"])
        np.testing.assert_array_equal(r["y"], plain[name + "_y"])


def test_solves_after_a_device_reset(cuda, tmp_path):
    """A caller that resets the device (cudaDeviceReset) between solves ends the context that
    owned the library's cached device blocks and page-locked records.  The cache keys blocks by
    the driver's context id and forgets those of an ended context, so the solves after the
    reset allocate afresh and give the results of the solves before it.  Runs in a child
    process (the reset would pull the device out from under this process's torch state); the
    child first checks through the driver that the reset gave the device a new context id."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    script = r'''
import ctypes, json, sys
import numpy as np
import vajra_pdhg as V
from vajra_pdhg import workloads as W
drv = ctypes.CDLL("libcuda.so.1")
def ctx_id():
    c = ctypes.c_void_p()
    assert drv.cuCtxGetCurrent(ctypes.byref(c)) == 0 and c.value
    i = ctypes.c_ulonglong()
    assert drv.cuCtxGetId(c, ctypes.byref(i)) == 0
    return i.value
lp = W.random_planted(300, 800, 6, seed=5)
before = V.solve(lp, precision=V.PREC_FP64)
batch_before = V.solve_batch([lp, lp], precision=V.PREC_FP64, autotune=0)
id0 = ctx_id()
rt = ctypes.CDLL("libcudart.so.12")
assert rt.cudaDeviceReset() == 0
assert rt.cudaFree(None) == 0
id1 = ctx_id()
if id1 == id0:
    print(json.dumps({"same_context": True}))
    sys.exit(3)
after = V.solve(lp, precision=V.PREC_FP64)
batch_after = V.solve_batch([lp, lp], precision=V.PREC_FP64, autotune=0)
out = {"status": [before["status_name"], after["status_name"]],
       "iterations": [before["iterations"], after["iterations"]],
       "x_equal": bool(np.array_equal(before["x"], after["x"])),
       "batch": [r["status_name"] for r in batch_after],
       "batch_x_equal": bool(np.array_equal(batch_before[0]["x"], batch_after[0]["x"]))}
print(json.dumps(out))
'''
    env = dict(os.environ,
               PYTHONPATH=os.pathsep.join([root, os.path.join(root, "vajra-opt_b200"), os.environ.get("PYTHONPATH", "")]))
    p = subprocess.run([sys.executable, "-c", script], env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-3000:]
    import json
    out = json.loads(p.stdout.strip().splitlines()[-1])
    assert out["status"] == ["OPTIMAL", "OPTIMAL"]
    assert out["iterations"][0] == out["iterations"][1] and out["x_equal"]
    assert out["batch"] == ["OPTIMAL", "OPTIMAL"] and out["batch_x_equal"]


def test_handover_default_follows_the_lp_size(cuda):
    """handover_mode = -1 (the default): below 2^20 entries the FP64 phase restarts from the
    FP32 candidate (the same solve as handover_mode = 0), from 2^20 entries on it continues the
    FP32 epoch (the same solve as handover_mode = 1)."""
    small = W.random_planted(2000, 5000, 8, seed=24)
    d, r = V.solve(small, precision=V.PREC_MIXED), V.solve(small, precision=V.PREC_MIXED, handover_mode=0)
    assert d["iterations"] == r["iterations"] and d["fp64_iterations"] == r["fp64_iterations"]
    np.testing.assert_array_equal(d["x"], r["x"])
    big = W.random_large(200_000, 400_000, seed=5)
    assert big.nnz >= 1 << 20
    kw = dict(precision=V.PREC_MIXED, spmv_shape_a=-3, spmv_shape_at=-3)
    d, c = V.solve(big, **kw), V.solve(big, handover_mode=1, **kw)
    assert d["status_name"] == "OPTIMAL" and d["fp32_iterations"] > 0
    assert d["iterations"] == c["iterations"] and d["fp64_iterations"] == c["fp64_iterations"]
    np.testing.assert_array_equal(d["x"], c["x"])
