"""VAJRA_ALGO_REFERENCE on the device vs the oracle (the reference CPU PDHG restated),
through vajra_pdhg_solve: vectors and diagnostics must be bit-identical."""
import numpy as np
import pytest

import vajra_pdhg as V
from oracle import bindings as B
from vajra_pdhg import workloads as W

pytestmark = pytest.mark.gpu
SCALARS = ("status", "iterations", "objective_value", "restart_count", "primal_residual", "dual_residual",
           "duality_gap", "spectral_norm_estimate", "tau", "sigma")
INF = 1e20


def run_both(lp, iters, cf=100, tol=1e-6, gap_tol=1e-6, scale=True, compare_col_dual=True):
    g = V.solve(lp, algorithm=V.ALGO_REFERENCE, iteration_limit=iters, check_frequency=cf, tolerance=tol,
                gap_tolerance=gap_tol, enable_scaling=int(scale))
    o = B.port_solve(lp, iteration_limit=iters, check_frequency=cf, tolerance=tol, gap_tolerance=gap_tol,
                     enable_scaling=scale)
    keys = ("x", "y", "row_value") + (("d",) if compare_col_dual else ())
    for k in keys:
        np.testing.assert_array_equal(g[k], o[k], err_msg=k)
    for k in SCALARS:
        assert g[k] == o[k] or (np.isnan(g[k]) and np.isnan(o[k])), (k, g[k], o[k])
    return g, o


def lp_from(rows, cols, trips, c, cl, cu, rl, ru, sense=0):
    from vajra_pdhg.workloads import canonical_csc, LP
    r = [t[0] for t in trips]; cc = [t[1] for t in trips]; v = [t[2] for t in trips]
    cp, ri, vals = canonical_csc(rows, cols, r, cc, v)
    return LP(rows, cols, cp, ri, vals, np.array(c, float), np.array(cl, float), np.array(cu, float),
              np.array(rl, float), np.array(ru, float), sense=sense)


@pytest.mark.parametrize("seed,m,n,k,iters,cf", [(1, 30, 70, 3, 2000, 100), (2, 50, 120, 5, 777, 7),
                                                 (3, 200, 500, 8, 3000, 100), (4, 2000, 5000, 8, 300, 100)])
def test_random_equality_bit_identical(cuda, seed, m, n, k, iters, cf):
    run_both(W.random_planted(m, n, k, seed=seed), iters, cf)


@pytest.mark.parametrize("seed", [3, 4, 5])
def test_mixed_senses_bit_identical(cuda, seed):
    run_both(W.small_random(40, 100, seed), 3000)


def test_without_scaling(cuda):
    run_both(W.small_random(25, 60, 4), 800, cf=50, scale=False)


def test_maximise_with_free_columns(cuda):
    lp = W.small_random(30, 60, 9)
    lp.sense = 1
    lp.c = -lp.c
    lp.col_lower = lp.col_lower.copy(); lp.col_upper = lp.col_upper.copy()
    lp.col_lower[::7] = -INF
    lp.col_upper[::7] = INF
    run_both(lp, 1500, compare_col_dual=False)


# The LPs of the reference's tests/test_pdhg.cpp, with their known optima.
PDHG_TEST_LPS = {
    "two_var_opt_-7": (lp_from(3, 2, [(0, 0, 1), (0, 1, 1), (1, 0, 1), (2, 1, 1)], [-1, -2], [0, 0], [INF, INF],
                               [-INF] * 3, [4, 3, 3]), -7.0, 1e-5, 20000),                       # :55-99
    "equality_13": (lp_from(2, 3, [(0, 0, 1), (0, 1, 1), (0, 2, 1), (1, 0, 2), (1, 1, 1)], [1, 2, 3], [0] * 3,
                            [INF] * 3, [6, 5], [6, 5]), 13.0, 1e-5, 20000),                      # :102-142
    "senses_4": (lp_from(3, 2, [(0, 0, 1), (0, 1, 1), (1, 0, 1), (1, 1, -1), (2, 0, 2), (2, 1, 1)], [2, 3], [0, 0],
                         [10, 10], [2, -INF, 1], [INF, 4, 6]), 4.0, 1e-5, 20000),                # :145-188
    "free_-5": (lp_from(1, 2, [(0, 0, 1), (0, 1, 1)], [2, 1], [-10, -INF], [10, INF], [5], [5]), -5.0, 1e-5, 20000),  # :191-231
    "min_-15": (lp_from(1, 2, [(0, 0, 1), (0, 1, 1)], [-2, -3], [0, 0], [INF, INF], [-INF], [5]), -15.0, 1e-5, 20000),  # :234-272
    "max_15": (lp_from(1, 2, [(0, 0, 1), (0, 1, 1)], [2, 3], [0, 0], [INF, INF], [-INF], [5], sense=1), 15.0, 1e-5, 20000),
    "gpu_request_3": (lp_from(1, 2, [(0, 0, 1), (0, 1, 1)], [1, 1], [0, 0], [10, 10], [3], [10]), 3.0, 1e-6, 5000),  # :405-436
}


@pytest.mark.parametrize("name", list(PDHG_TEST_LPS))
def test_reference_test_lps(cuda, name):
    lp, opt, tol, iters = PDHG_TEST_LPS[name]
    g, o = run_both(lp, iters, tol=tol, compare_col_dual=(lp.sense == 0))
    if g["status_name"] == "OPTIMAL":
        assert abs(g["objective_value"] - opt) <= 1e-3


def test_infeasible_is_not_optimal(cuda):
    lp = lp_from(2, 2, [(0, 0, 1), (0, 1, 1), (1, 0, 1), (1, 1, 1)], [1, 1], [0, 0], [10, 10], [-INF, 3], [1, INF])
    g, _ = run_both(lp, 500)                                  # test_pdhg.cpp:317-348
    assert g["status_name"] != "OPTIMAL"


def test_iteration_limit_zero_and_small(cuda):
    lp = W.random_planted(20, 50, 3, seed=8)
    g, _ = run_both(lp, 0)
    assert g["status_name"] == "ITERATION_LIMIT" and g["iterations"] == 1
    g, _ = run_both(lp, 10)
    assert g["status_name"] in ("ITERATION_LIMIT", "FEASIBLE") and g["iterations"] == 11


def test_nan_in_objective_is_numerical_error(cuda):
    lp = W.random_planted(20, 50, 3, seed=9)
    lp.c = lp.c.copy(); lp.c[5] = np.nan
    g, _ = run_both(lp, 100)
    assert g["status_name"] == "NUMERICAL_ERROR" and g["iterations"] == 1


def test_nan_in_matrix_is_numerical_error(cuda):
    lp = W.random_planted(20, 50, 3, seed=10)
    lp.values = lp.values.copy(); lp.values[7] = np.nan
    g, _ = run_both(lp, 100)
    assert g["status_name"] == "NUMERICAL_ERROR"


def test_repeated_runs_are_deterministic(cuda):
    lp = W.random_planted(100, 250, 5, seed=12)
    with V.Solver(lp, algorithm=V.ALGO_REFERENCE, iteration_limit=1000) as s:
        a, b = s.run(), s.run()
    for k in ("x", "y", "d", "row_value"):
        np.testing.assert_array_equal(a[k], b[k])
    assert a["iterations"] == b["iterations"]
