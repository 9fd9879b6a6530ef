"""The seeded synthetic workloads that stand in for the benchmark configurations: canonical CSC
(rows ascending and unique within a column, |v| <= 1e-11 dropped, duplicates summed), the
planted optima they claim, and the shapes the configurations name."""
import numpy as np
import pytest

from vajra_pdhg import workloads as W
from vajra_pdhg.kkt import relative_kkt


def assert_canonical(lp):
    cp, ri = lp.col_ptr, lp.row_idx
    assert cp[0] == 0 and cp[-1] == lp.nnz and np.all(np.diff(cp) >= 0)
    assert ri.min(initial=0) >= 0 and ri.max(initial=-1) < lp.num_rows
    for j in range(lp.num_cols):
        seg = ri[cp[j]:cp[j + 1]]
        assert np.all(np.diff(seg) > 0), j
    assert np.all(np.abs(lp.values) > 1e-11)


def test_canonical_csc_sums_duplicates_and_drops_tiny_values():
    cp, ri, v = W.canonical_csc(3, 2, [2, 0, 2, 1, 1], [0, 0, 0, 1, 1], [1.0, 2.0, 3.0, 1e-12, 5.0])
    assert list(cp) == [0, 2, 3]
    assert list(ri) == [0, 2, 1]
    assert list(v) == [2.0, 4.0, 5.0]


def test_random_planted_optimum_is_primal_dual_optimal():
    lp = W.random_planted(200, 500, 8, seed=0)
    assert_canonical(lp)
    k = relative_kkt(lp, lp.x_planted, lp.y_planted)
    assert k["rel_kkt"] <= 1e-12, k
    assert k["primal_objective"] == pytest.approx(lp.planted_objective, rel=1e-12)


def test_random_large_shape_at_reduced_size():
    lp = W.random_large(20000, 40000, seed=1)
    assert_canonical(lp)
    deg = np.diff(lp.col_ptr)
    assert deg.max() <= 2000 and deg.min() >= 1
    assert 8.0 < deg.mean() < 12.0                       # mean 10 before duplicates merge
    assert np.all(lp.values == lp.values.astype(np.float32))   # stored FP32-exact
    eq = lp.row_lower == lp.row_upper
    assert 0.65 < eq.mean() < 0.75                       # 70 % equality rows
    k = relative_kkt(lp, lp.x_planted, lp.y_planted)
    assert k["rel_kkt"] <= 1e-12, k


def test_min_cost_flow_is_an_incidence_matrix():
    lp = W.min_cost_flow(nodes=500, arcs=3000, seed=2)
    assert_canonical(lp)
    assert np.all(np.diff(lp.col_ptr) == 2)
    v = lp.values.reshape(-1, 2)
    assert np.all(np.sort(v, axis=1) == [-1.0, 1.0])
    assert np.all(lp.row_lower == lp.row_upper)
