"""FP64 relative KKT report of a primal-dual point on the original (unscaled) LP, on the host.

Independent of the device code: it is how tests and the benchmark check the device's own
KKT figure.  Definitions (minimisation form; a maximisation LP is negated first):

  rel_primal = ||A x - proj_[row_lower,row_upper](A x)||_2 / (1 + ||b||_2)
  rel_dual   = ||r - lambda||_2 / (1 + ||c||_2),  r = c - A^T y,  lambda = the part of r the
               column bounds allow (r where both bounds are finite, max(r,0) with only a lower
               bound, min(r,0) with only an upper bound, 0 for a free column)
  rel_gap    = |pobj - dobj| / (1 + |pobj| + |dobj|), with the dual objective of
               src/solvers/pdhg/pdhg.cpp:279-313 evaluated at (y, lambda)
  rel_kkt    = max of the three

||b|| counts every finite row bound, an equality row once.  y is the row dual of the
minimisation form in the verifier's sign convention (<= row: y <= 0, >= row: y >= 0) for both
objective senses, as VAJRA_ALGO_HALPERN returns it in vajra_result.row_dual.
"""
from __future__ import annotations

import numpy as np

INF = 1e20


def bound_norm(lp) -> float:
    """||b||_2 of the relative KKT: every finite row bound, an equality row once."""
    rl, ru = np.asarray(lp.row_lower, float), np.asarray(lp.row_upper, float)
    rlf, ruf = rl > -INF, ru < INF
    eq = rlf & ruf & (rl == ru)
    b2 = np.where(eq, rl ** 2, np.where(rlf, rl, 0.0) ** 2 + np.where(ruf, ru, 0.0) ** 2)
    return float(np.sqrt(b2.sum()))


def relative_kkt(lp, x, row_dual) -> dict:
    A = lp.to_scipy_csc()
    is_max = int(getattr(lp, "sense", 0)) != 0
    c = -np.asarray(lp.c, float) if is_max else np.asarray(lp.c, float)
    y = np.asarray(row_dual, float)
    off = float(getattr(lp, "objective_offset", 0.0))
    off = -off if is_max else off
    rl, ru = np.asarray(lp.row_lower, float), np.asarray(lp.row_upper, float)
    cl, cu = np.asarray(lp.col_lower, float), np.asarray(lp.col_upper, float)
    x = np.asarray(x, float)
    ax = A @ x
    rp = ax - np.clip(ax, rl, ru)
    r = c - A.T @ y
    lf, uf = cl > -INF, cu < INF
    lam = np.where(lf & uf, r, np.where(lf, np.maximum(r, 0.0), np.where(uf, np.minimum(r, 0.0), 0.0)))
    rd = r - lam
    rlf, ruf = rl > -INF, ru < INF
    dobj = np.sum(np.where((y > 0) & rlf, y * np.where(rlf, rl, 0.0), 0.0))
    dobj += np.sum(np.where((y < 0) & ruf, y * np.where(ruf, ru, 0.0), 0.0))
    dobj += np.sum(np.where(lam > 0, lam * np.where(lf, cl, 0.0), lam * np.where(uf, cu, 0.0))) + off
    pobj = float(c @ x) + off
    rel_p = float(np.linalg.norm(rp) / (1.0 + bound_norm(lp)))
    rel_d = float(np.linalg.norm(rd) / (1.0 + np.linalg.norm(np.asarray(lp.c, float))))
    rel_gap = float(abs(pobj - dobj) / (1.0 + abs(pobj) + abs(dobj)))
    return {"rel_primal": rel_p, "rel_dual": rel_d, "rel_gap": rel_gap, "rel_kkt": max(rel_p, rel_d, rel_gap),
            "primal_objective": pobj, "dual_objective": dobj,
            "max_row_violation": float(np.max(np.abs(rp), initial=0.0)),
            "max_bound_violation": float(max(np.max(cl - x, initial=0.0), np.max(x - cu, initial=0.0)))}


def guard_maxima(lp, x, row_dual) -> dict:
    """The quantities the engine's status guard checks on a returned point
    (Solution::recompute_quality, src/engine/model.cpp:203-374, LP part; 1e-7 thresholds of
    include/indus/tolerances.hpp): the largest row violation over 1 + |violated bound| and its
    absolute size, and the largest reduced-cost / row-dual sign violation (minimisation form,
    verifier sign convention)."""
    A = lp.to_scipy_csc()
    is_max = int(getattr(lp, "sense", 0)) != 0
    c = -np.asarray(lp.c, float) if is_max else np.asarray(lp.c, float)
    x = np.asarray(x, float)
    y = np.asarray(row_dual, float)
    rl, ru = np.asarray(lp.row_lower, float), np.asarray(lp.row_upper, float)
    cl, cu = np.asarray(lp.col_lower, float), np.asarray(lp.col_upper, float)
    ax = A @ x
    below = np.maximum(rl - ax, 0.0)
    above = np.maximum(ax - ru, 0.0)
    den_b = 1.0 + np.where(rl > -1e19, np.abs(rl), 1.0)
    den_a = 1.0 + np.where(ru < 1e19, np.abs(ru), 1.0)
    p_rel = float(max(np.max(below / den_b, initial=0.0), np.max(above / den_a, initial=0.0)))
    p_abs = float(max(np.max(below, initial=0.0), np.max(above, initial=0.0)))
    d = c - A.T @ y
    t = 1e-7
    dv = np.maximum(np.where((x < cu - t) & (d < 0), -d, 0.0), np.where((x > cl + t) & (d > 0), d, 0.0))
    le = (rl <= -1e20) & (ru < 1e20)
    ge = (rl > -1e20) & (ru >= 1e20)
    yv = np.maximum(np.where(le & (y > 0), y, 0.0), np.where(ge & (y < 0), -y, 0.0))
    return {"primal_rel": p_rel, "primal_abs": p_abs,
            "dual_abs": float(max(np.max(dv, initial=0.0), np.max(yv, initial=0.0)))}
