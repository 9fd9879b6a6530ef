"""The device set-up's scaling (vajra_scale_lp) against the reference's own host scaling,
compiled from its sources into oracle/_ref:

* Ruiz alone: RuizScaler::compute_and_scale (src/linalg/scaling.cpp:7-153), bit for bit --
  factors, scaled values, scaled c and bounds;
* Ruiz, then Pock-Chambolle: PockChambollePreconditioner::compute (scaling.cpp:179-220, alpha =
  1) on the Ruiz-scaled matrix, applied as A <- diag(sqrt(d_row)) A diag(sqrt(d_col)).  The
  device sums |a| in the reference's order (bit-exact sums) and forms 1/sqrt(s) where the
  reference forms d = 1/s; sqrt(1/s) and 1/sqrt(s), each a sequence of two correctly rounded
  operations, differ by at most two units in the last place, so the factors and everything
  scaled by them agree to a few ulps, not bit for bit.
"""
import numpy as np
import pytest

import vajra_pdhg as V
from oracle import bindings as B
from vajra_pdhg import workloads as W

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not B.ref_available(), reason="needs oracle/_ref")]
INF = 1e20
ULPS = 8 * np.finfo(np.float64).eps


def lps():
    a = W.small_random(300, 700, 41)
    b = W.small_random(150, 400, 9)
    b.sense = 1
    b.c = -b.c
    b.col_lower = b.col_lower.copy()
    b.col_lower[::11] = -INF
    c = W.random_planted(500, 1300, (2, 30), seed=42)
    return [a, b, c]


def scaled_bounds(v, scale, rows):
    """Finite bounds times the row scale / divided by the column scale (scaling.cpp:104-149)."""
    out = v.copy()
    fin = np.abs(v) < INF
    out[fin] = v[fin] * scale[fin] if rows else v[fin] * (1.0 / scale[fin])
    return out


@pytest.mark.parametrize("k", range(3))
def test_ruiz_alone_is_bit_identical(cuda, k):
    lp = lps()[k]
    d = V.scale_lp(lp, pock_chambolle=0)
    r = B.ref_ruiz(lp)
    for key in ("row_scale", "col_scale", "values", "row_lower", "row_upper", "col_lower", "col_upper"):
        np.testing.assert_array_equal(d[key], r[key], err_msg=key)
    np.testing.assert_array_equal(d["c"], -r["c"] if lp.sense else r["c"])


@pytest.mark.parametrize("k", range(3))
def test_ruiz_then_pock_chambolle_matches_the_reference(cuda, k):
    lp = lps()[k]
    d = V.scale_lp(lp, pock_chambolle=1)
    r = B.ref_ruiz(lp)
    ruized = W.LP(**{**lp.__dict__})
    ruized.values = r["values"]
    d_row, d_col = B.ref_pock_chambolle(ruized, 1.0)
    pr, pc = np.sqrt(d_row), np.sqrt(d_col)
    rows = np.asarray(lp.row_idx)
    cols = np.repeat(np.arange(lp.num_cols), np.diff(lp.col_ptr))
    want = {"row_scale": r["row_scale"] * pr, "col_scale": r["col_scale"] * pc,
            "values": r["values"] * (pr[rows] * pc[cols])}
    for key, v in want.items():
        np.testing.assert_allclose(d[key], v, rtol=ULPS, atol=0, err_msg=key)
    c = r["c"] * pc
    np.testing.assert_allclose(d["c"], -c if lp.sense else c, rtol=ULPS, atol=0)
    np.testing.assert_allclose(d["row_lower"], scaled_bounds(np.asarray(lp.row_lower, float), want["row_scale"], True),
                               rtol=ULPS, atol=0)
    np.testing.assert_allclose(d["col_upper"], scaled_bounds(np.asarray(lp.col_upper, float), want["col_scale"], False),
                               rtol=ULPS, atol=0)


def test_one_ruiz_pass_then_pock_chambolle(cuda):
    """A single Ruiz pass (the factors far from converged) followed by Pock-Chambolle."""
    lp = lps()[0]
    d = V.scale_lp(lp, pock_chambolle=1, ruiz_iterations=1)
    r = B.ref_ruiz(lp, max_iters=1)
    ruized = W.LP(**{**lp.__dict__})
    ruized.values = r["values"]
    d_row, d_col = B.ref_pock_chambolle(ruized, 1.0)
    np.testing.assert_allclose(d["row_scale"], r["row_scale"] * np.sqrt(d_row), rtol=ULPS, atol=0)
    np.testing.assert_allclose(d["col_scale"], r["col_scale"] * np.sqrt(d_col), rtol=ULPS, atol=0)
