"""Adjoint of the unrolled PDHG map (vajra_pdhg_unrolled) against FP64 finite differences of
the same map (kink-aware), checkpoint invariance, the torch.autograd harness, and the
optimal-value gradient dV/db = y* against the reference's own dual simplex."""
import numpy as np
import pytest

from oracle import bindings as B
from vajra_pdhg import workloads as W
from vajra_pdhg.autograd import PREC_FP32, PREC_FP64, PREC_MIXED, unrolled

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


def fd_central(lps, w, dc, db, h, **opts):
    """FP64 central differences of sum_i L_i along (dc, db) at steps h and h/2.

    L = (w + c).x(K) is quadratic in c on top of the unrolled map, which is piecewise affine in
    (c, b) (every step is affine up to the bound projections).  Where no projection changes its
    active set within +-h the function is a quadratic along the line, so the central
    difference is exact and does not depend on the step: the two agree to rounding.  A
    disagreement flags an active-set change (a kink) within +-h."""
    def total(t):
        cs = split(lps, packed(lps, "c") + t * dc, rows=False)
        bs = split(lps, packed(lps, "row_lower") + t * db, rows=True)
        pert = [with_cb(lp, c, b) for lp, c, b in zip(lps, cs, bs)]
        return unrolled(pert, w, gradients=False, precision=PREC_FP64, **opts)["loss"].sum()
    return (total(h) - total(-h)) / (2 * h), (total(h / 2) - total(-h / 2)) / h


@pytest.mark.parametrize("prec,tol", [(PREC_FP64, 1e-6), (PREC_MIXED, 1e-4)])
def test_adjoint_matches_fp64_finite_differences(cuda, prec, tol):
    """Every direction without an active-set change within +-h (central differences at h and
    h/2 agree) must match the adjoint to `tol`; only kink-flagged directions may miss."""
    lps = batch()
    rng = np.random.default_rng(1)
    N = sum(lp.num_cols for lp in lps)
    M = sum(lp.num_rows for lp in lps)
    w = rng.standard_normal(N)
    opts = dict(iterations=300, checkpoint_every=50)
    g = unrolled(lps, w, precision=prec, **opts)
    gb = g["grad_row_lower"] + g["grad_row_upper"]
    clean, flagged = [], 0
    for _ in range(16):
        dc = rng.standard_normal(N)
        db = rng.standard_normal(M)
        adj = g["grad_c"] @ dc + gb @ db
        c1, c2 = fd_central(lps, w, dc, db, 1e-6, **opts)
        if abs(c1 - c2) <= 1e-7 * abs(c1):
            clean.append(abs(adj - c1) / max(1e-12, abs(c1)))
        else:
            flagged += 1
    assert len(clean) >= 8, (clean, flagged)
    assert max(clean) <= tol, clean


def test_fp32_map_adjoint_against_fp64_differences(cuda):
    """The pure FP32 map (PREC_FP32): its derivative differs from the FP64 map's where an active
    set flipped between the two maps; on this short map it still matches to 1e-3 (median)."""
    lps = batch()
    rng = np.random.default_rng(5)
    N = sum(lp.num_cols for lp in lps)
    M = sum(lp.num_rows for lp in lps)
    w = rng.standard_normal(N)
    opts = dict(iterations=300, checkpoint_every=50)
    g = unrolled(lps, w, precision=PREC_FP32, **opts)
    gb = g["grad_row_lower"] + g["grad_row_upper"]
    errs = []
    for _ in range(8):
        dc = rng.standard_normal(N)
        db = rng.standard_normal(M)
        adj = g["grad_c"] @ dc + gb @ db
        c1, _ = fd_central(lps, w, dc, db, 1e-6, **opts)
        errs.append(abs(adj - c1) / max(1e-12, abs(c1)))
    assert np.median(errs) <= 1e-3, errs


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
@pytest.mark.parametrize("m,n,k,seed", [(60, 150, 5, 44), (200, 500, 8, 47)])
def test_optimal_value_gradient_matches_simplex_duals(cuda, m, n, k, seed):
    """dV/db of V(c, b) = min c.x (the OptimalValue harness: the restarted Halpern solver to
    FP64 relative KKT 1e-10, envelope-theorem backward) against the reference dual simplex's
    y* (src/engine/model.cpp:528-614) to 1e-4, and against central differences of V itself.
    y* is unique when the columns strictly between their bounds at the planted optimum have
    full row rank (checked first: otherwise two correct solvers may return different duals)."""
    import torch
    from vajra_pdhg.autograd import OptimalValue
    lp = W.random_planted(m, n, k, seed=seed)
    interior = (lp.x_planted > 1e-9) & (lp.x_planted < 10 - 1e-9)
    assert np.linalg.matrix_rank(lp.to_scipy_csc()[:, np.flatnonzero(interior)].toarray()) == m
    s = B.ref_solve(lp, algorithm="dual_simplex", through_solve=True, iteration_limit=100000)
    assert s["status_name"] == "OPTIMAL"
    c = torch.tensor(lp.c, dtype=torch.float64, requires_grad=True)
    b = torch.tensor(lp.row_lower, dtype=torch.float64, requires_grad=True)
    v = OptimalValue.apply(c, b, [lp], None)
    v.sum().backward()
    y = b.grad.numpy()
    assert abs(v.item() - s["objective_value"]) <= 1e-8 * (1 + abs(s["objective_value"]))
    assert np.linalg.norm(y - s["y"]) <= 1e-4 * np.linalg.norm(s["y"]), np.linalg.norm(y - s["y"])
    # V is piecewise linear in b: central differences along a few directions
    rng = np.random.default_rng(seed)
    h = 1e-5 * np.linalg.norm(lp.row_lower)
    for _ in range(3):
        d = rng.standard_normal(m)
        d /= np.linalg.norm(d)
        vp = OptimalValue.apply(c.detach(), b.detach() + h * torch.from_numpy(d), [lp], None).item()
        vm = OptimalValue.apply(c.detach(), b.detach() - h * torch.from_numpy(d), [lp], None).item()
        fd = (vp - vm) / (2 * h)
        assert abs(fd - y @ d) <= 1e-4 * np.linalg.norm(y), (fd, y @ d)
