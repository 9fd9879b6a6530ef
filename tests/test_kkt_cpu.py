"""The host FP64 relative KKT (vajra_pdhg/kkt.py), the yardstick every solver result is checked
against: zero at known optima of both senses, the primal part equal to the row violation,
||b|| counting each equality row once, and small at HiGHS optima of random LPs, where the
reference's own verifier agrees."""
import numpy as np
import pytest
import scipy.optimize as so

from oracle import bindings as B
from vajra_pdhg import workloads as W
from vajra_pdhg.kkt import bound_norm, relative_kkt

INF = 1e20


def lp_from(m, n, trips, c, cl, cu, rl, ru, sense=0):
    cp, ri, vals = W.canonical_csc(m, n, [t[0] for t in trips], [t[1] for t in trips], [t[2] for t in trips])
    return W.LP(m, n, cp, ri, vals, np.array(c, float), np.array(cl, float), np.array(cu, float),
                np.array(rl, float), np.array(ru, float), sense=sense)


def test_zero_at_a_known_minimum():
    # min x0 + 2 x1  s.t.  x0 + x1 >= 1,  0 <= x <= 10:  x* = (1, 0), y* = 1 (>= row: y >= 0)
    lp = lp_from(1, 2, [(0, 0, 1.0), (0, 1, 1.0)], [1, 2], [0, 0], [10, 10], [1], [INF])
    k = relative_kkt(lp, [1.0, 0.0], [1.0])
    assert k["rel_kkt"] == 0.0
    assert k["primal_objective"] == 1.0 and k["dual_objective"] == 1.0


def test_zero_at_a_known_maximum():
    # max x0 + x1  s.t.  x0 + x1 <= 3,  x >= 0: minimisation form min -x0 - x1, y* = -1 (<= row)
    lp = lp_from(1, 2, [(0, 0, 1.0), (0, 1, 1.0)], [1, 1], [0, 0], [INF, INF], [-INF], [3], sense=1)
    k = relative_kkt(lp, [1.5, 1.5], [-1.0])
    assert k["rel_kkt"] == 0.0
    assert k["primal_objective"] == -3.0


def test_primal_part_is_the_row_violation():
    lp = lp_from(2, 2, [(0, 0, 1.0), (1, 1, 1.0)], [1, 1], [0, 0], [10, 10], [1, 2], [1, 5])
    k = relative_kkt(lp, [0.5, 7.0], [0.0, 0.0])
    # rows: x0 = 0.5 against [1, 1] (0.5 short), x1 = 7 against [2, 5] (2 over)
    assert k["rel_primal"] == pytest.approx(np.hypot(0.5, 2.0) / (1.0 + bound_norm(lp)), rel=1e-15)
    assert k["max_row_violation"] == 2.0


def test_bound_norm_counts_an_equality_row_once():
    lp = lp_from(3, 1, [(0, 0, 1.0), (1, 0, 1.0), (2, 0, 1.0)], [0], [0], [1], [2, -INF, 1], [2, 3, 4])
    assert bound_norm(lp) == pytest.approx(np.sqrt(2 ** 2 + 3 ** 2 + 1 ** 2 + 4 ** 2), rel=1e-15)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_small_at_highs_optima(seed):
    rng = np.random.default_rng(seed)
    m, n = 40, 90
    A = rng.normal(size=(m, n)) * (rng.random((m, n)) < 0.15)
    x0 = rng.uniform(0, 5, n)
    eq = rng.random(m) < 0.5
    b = A @ x0
    ub = np.where(eq, b, b + rng.uniform(0.1, 1.0, m))
    c = rng.normal(size=n)
    res = so.linprog(c, A_ub=A[~eq], b_ub=ub[~eq], A_eq=A[eq], b_eq=b[eq], bounds=[(0, 5)] * n, method="highs")
    assert res.status == 0
    rows, cols = np.nonzero(A)
    lp = lp_from(m, n, list(zip(rows, cols, A[rows, cols])), c, np.zeros(n), np.full(n, 5.0),
                 np.where(eq, b, -INF), ub)
    # scipy's marginals are d(objective)/d(b): the row duals in the verifier's convention
    y = np.zeros(m)
    y[eq] = res.eqlin.marginals
    y[~eq] = res.ineqlin.marginals
    k = relative_kkt(lp, res.x, y)
    assert k["rel_kkt"] <= 1e-7, k
    if B.ref_available():
        v = B.ref_verify(lp, res.x, y, res.fun, 1, tol=1e-6)
        assert v["passed"], v["summary"]
