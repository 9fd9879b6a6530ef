"""Adjoint of the unrolled PDHG map (vajra_pdhg_unrolled) against FP64 one-sided finite
differences of the same map (kink-aware), checkpoint invariance, the torch.autograd harness,
and the optimal-value gradient y* = dV/db from the reference's own dual simplex."""
import numpy as np
import pytest

from oracle import bindings as B
from vajra_pdhg import workloads as W
from vajra_pdhg.autograd import PREC_FP64, PREC_MIXED, unrolled

pytestmark = pytest.mark.gpu


def batch(count=4, m=40, n=100, seed=0):
    return [W.random_planted(m, n, 4, seed=seed * 100 + i) for i in range(count)]


def with_cb(lp, c, b):
    out = W.LP(**{**lp.__dict__})
    out.c = c
    out.row_lower = b.copy()
    out.row_upper = b.copy()
    return out


def packed(lps, key):
    return np.concatenate([np.asarray(getattr(lp, key), float) for lp in lps])


def split(lps, vec, rows):
    out, o = [], 0
    for lp in lps:
        k = lp.num_rows if rows else lp.num_cols
        out.append(vec[o:o + k])
        o += k
    return out


def fd_directional(lps, w, dc, db, h, **opts):
    """FP64 one-sided differences of sum_i L_i along (dc, db): (forward, backward).

    The unrolled map is piecewise affine in (c, b) (every step is affine up to the bound
    projections).  The derivative at 0 equals the one-sided difference on any side whose
    interval (0, +-h] holds no change of a projection's active set, so a correct adjoint
    matches at least one of the two unless both sides hold one."""
    def total(sign):
        cs = split(lps, packed(lps, "c") + sign * h * dc, rows=False)
        bs = split(lps, packed(lps, "row_lower") + sign * h * db, rows=True)
        pert = [with_cb(lp, c, b) for lp, c, b in zip(lps, cs, bs)]
        return unrolled(pert, w, gradients=False, precision=PREC_FP64, **opts)["loss"].sum()
    f0 = total(0)
    return (total(+1) - f0) / h, (f0 - total(-1)) / h


@pytest.mark.parametrize("prec,tol", [(PREC_FP64, 1e-6), (PREC_MIXED, 1e-4)])
def test_adjoint_matches_fp64_finite_differences(cuda, prec, tol):
    lps = batch()
    rng = np.random.default_rng(1)
    N = sum(lp.num_cols for lp in lps)
    M = sum(lp.num_rows for lp in lps)
    w = rng.standard_normal(N)
    opts = dict(iterations=300, checkpoint_every=50)
    g = unrolled(lps, w, precision=prec, **opts)
    gb = g["grad_row_lower"] + g["grad_row_upper"]
    errs, misses = [], []
    while len(errs) < 8:
        # a wrong adjoint misses in every direction; a kink on both sides of 0 is rare
        assert len(misses) <= 4, (errs, misses)
        dc = rng.standard_normal(N)
        db = rng.standard_normal(M)
        adj = g["grad_c"] @ dc + gb @ db
        e = min(abs(adj - fd) / max(1e-12, abs(fd)) for fd in fd_directional(lps, w, dc, db, 1e-7, **opts))
        (errs if e <= tol else misses).append(e)
    assert max(errs) <= tol, errs


def test_checkpoint_interval_does_not_change_gradients(cuda):
    lps = batch(count=3, seed=2)
    w = np.random.default_rng(2).standard_normal(sum(lp.num_cols for lp in lps))
    ref = unrolled(lps, w, iterations=120, checkpoint_every=120, precision=PREC_MIXED)
    for ck in (1, 7, 50):
        g = unrolled(lps, w, iterations=120, checkpoint_every=ck, precision=PREC_MIXED)
        for k in ("loss", "x", "grad_c", "grad_row_lower", "grad_row_upper"):
            np.testing.assert_array_equal(g[k], ref[k], err_msg=f"{k} at checkpoint {ck}")


def test_autograd_function(cuda):
    import torch
    from vajra_pdhg.autograd import UnrolledLoss
    lps = batch(count=3, seed=3)
    c = torch.tensor(packed(lps, "c"), requires_grad=True)
    b = torch.tensor(packed(lps, "row_lower"), requires_grad=True)
    w = torch.randn(c.numel(), dtype=torch.float64)
    opts = dict(iterations=200, checkpoint_every=40, precision=PREC_FP64)
    loss = UnrolledLoss.apply(c, b, lps, w, opts)
    (loss * torch.tensor([1.0, 2.0, -0.5], dtype=torch.float64)).sum().backward()
    g = unrolled(lps, w.numpy(), **opts)
    col_scale = np.repeat([1.0, 2.0, -0.5], [lp.num_cols for lp in lps])
    row_scale = np.repeat([1.0, 2.0, -0.5], [lp.num_rows for lp in lps])
    np.testing.assert_allclose(c.grad.numpy(), g["grad_c"] * col_scale, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(b.grad.numpy(), (g["grad_row_lower"] + g["grad_row_upper"]) * row_scale,
                               rtol=1e-12, atol=1e-12)


@pytest.mark.skipif(not B.ref_available(), reason="needs the reference's dual simplex (oracle/_ref)")
def test_objective_gradient_wrt_b_approaches_simplex_duals(cuda):
    """dV/db = y* (unique here); the unrolled map's derivative of c.x(K) approaches it as K
    grows (slowly: the plain unrolled iteration has no restarts)."""
    lp = W.random_planted(60, 150, 5, seed=44)
    s = B.ref_solve(lp, algorithm="dual_simplex", through_solve=True, iteration_limit=100000)
    assert s["status_name"] == "OPTIMAL"
    rel = {}
    for k in (5000, 20000):
        g = unrolled([lp], None, iterations=k, checkpoint_every=500, precision=PREC_FP64)
        gb = g["grad_row_lower"] + g["grad_row_upper"]
        rel[k] = np.linalg.norm(gb - s["y"]) / np.linalg.norm(s["y"])
    assert rel[20000] < rel[5000] and rel[20000] <= 0.05, rel
