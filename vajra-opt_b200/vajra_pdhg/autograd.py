"""Gradient harnesses: the adjoint of the unrolled PDHG map (vajra_pdhg_unrolled) and the
gradient of the optimal value at a converged solution.

`unrolled(lps, weights, ...)` calls the C ABI directly.  `UnrolledLoss` is a thin
torch.autograd.Function around it: forward returns the per-instance losses
L_i = sum_j (w_j + c_j) x_j(K), backward applies the device adjoint's dL/dc and dL/db (for
equality rows b = row_lower = row_upper, so dL/db = dL/drow_lower + dL/drow_upper).

`OptimalValue` differentiates V(c, b) = min {c.x : A x = b, l <= x <= u} itself: forward solves
each LP to a tight FP64 relative KKT with the restarted Halpern solver, backward returns the
envelope-theorem gradient dV/dc = x*, dV/db = y* (the row dual in the verifier's convention,
col_dual = c - A^T y), which is exact wherever the optimal basis is unique.  torch is used only
to carry tensors through autograd; all arithmetic runs in libvajra_pdhg.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi, _HostLp
from ._capi import PREC_FP32, PREC_FP64, PREC_MIXED


class VajraUnrolledOpts(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("checkpoint_every", C.c_int32), ("precision", C.c_int32),
                ("enable_scaling", C.c_int32), ("step_safety", C.c_double), ("device", C.c_int32),
                ("reserved", C.c_int32 * 5)]


def default_unrolled_opts(**overrides) -> VajraUnrolledOpts:
    o = VajraUnrolledOpts()
    _capi.lib().vajra_default_unrolled_opts(C.byref(o))
    for k, v in overrides.items():
        if not hasattr(o, k):
            raise KeyError(f"unknown option {k!r}")
        setattr(o, k, v)
    return o


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def unrolled(lps, weights=None, gradients=True, **opts) -> dict:
    """Loss per instance, final iterate and (optionally) the adjoint gradients, packed in
    instance order (N = sum of columns, M = sum of rows)."""
    hosts = [_HostLp(lp) for lp in lps]
    arr = (_capi.VajraLp * len(lps))(*[h.s for h in hosts])
    N = sum(int(lp.num_cols) for lp in lps)
    M = sum(int(lp.num_rows) for lp in lps)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    if w is not None and w.size != N:
        raise ValueError(f"weights has {w.size} entries, expected {N}")
    out = {"loss": np.zeros(len(lps)), "x": np.zeros(N)}
    if gradients:
        out.update(grad_c=np.zeros(N), grad_row_lower=np.zeros(M), grad_row_upper=np.zeros(M))
    o = default_unrolled_opts(**opts)
    st = _capi.lib().vajra_pdhg_unrolled(len(lps), C.cast(arr, C.c_void_p), C.cast(C.pointer(o), C.c_void_p),
                                         _dp(w), _dp(out["loss"]), _dp(out["x"]), _dp(out.get("grad_c")),
                                         _dp(out.get("grad_row_lower")), _dp(out.get("grad_row_upper")))
    if st != _capi.OK:
        raise RuntimeError(f"vajra_pdhg_unrolled failed: status {st} "
                           f"({_capi.lib().vajra_status_string(st).decode()})")
    return out


def _with_cb(template, c, b):
    """Copy of an equality-row LP with objective c and right-hand side b."""
    from .workloads import LP
    return LP(template.num_rows, template.num_cols, template.col_ptr, template.row_idx, template.values,
              np.asarray(c, dtype=np.float64), template.col_lower, template.col_upper,
              np.asarray(b, dtype=np.float64).copy(), np.asarray(b, dtype=np.float64).copy())


try:
    import torch

    class UnrolledLoss(torch.autograd.Function):
        """L(c, b) per instance for equality-constrained LPs sharing A and bounds with `templates`."""

        @staticmethod
        def forward(ctx, c, b, templates, weights, opts):
            cs = c.detach().cpu().double().numpy()
            bs = b.detach().cpu().double().numpy()
            lps, co, ro = [], 0, 0
            for t in templates:
                lps.append(_with_cb(t, cs[co:co + t.num_cols], bs[ro:ro + t.num_rows]))
                co += t.num_cols
                ro += t.num_rows
            w = None if weights is None else weights.detach().cpu().double().numpy()
            r = unrolled(lps, w, gradients=True, **(opts or {}))
            ctx.grad_c = torch.from_numpy(r["grad_c"])
            ctx.grad_b = torch.from_numpy(r["grad_row_lower"] + r["grad_row_upper"])
            ctx.col_inst = torch.repeat_interleave(torch.arange(len(templates)),
                                                   torch.tensor([t.num_cols for t in templates]))
            ctx.row_inst = torch.repeat_interleave(torch.arange(len(templates)),
                                                   torch.tensor([t.num_rows for t in templates]))
            return torch.from_numpy(r["loss"]).to(c.device)

        @staticmethod
        def backward(ctx, g):
            g = g.detach().cpu().double()
            gc = ctx.grad_c * g[ctx.col_inst]
            gb = ctx.grad_b * g[ctx.row_inst]
            return gc, gb, None, None, None

    class OptimalValue(torch.autograd.Function):
        """V_i(c, b) per instance for equality-constrained LPs sharing A and bounds with
        `templates`; backward: dV/dc = x*, dV/db = y* at the solutions forward found."""

        @staticmethod
        def forward(ctx, c, b, templates, solve_opts):
            from . import solve
            cs = c.detach().cpu().double().numpy()
            bs = b.detach().cpu().double().numpy()
            vals, xs, ys, co, ro = [], [], [], 0, 0
            opts = {"precision": PREC_FP64, "tolerance": 1e-10, **(solve_opts or {})}
            for t in templates:
                r = solve(_with_cb(t, cs[co:co + t.num_cols], bs[ro:ro + t.num_rows]), **opts)
                if r["status_name"] != "OPTIMAL":
                    raise RuntimeError(f"OptimalValue: instance solve ended {r['status_name']}")
                vals.append(r["objective_value"])
                xs.append(r["x"])
                ys.append(r["y"])
                co += t.num_cols
                ro += t.num_rows
            ctx.x = torch.from_numpy(np.concatenate(xs))
            ctx.y = torch.from_numpy(np.concatenate(ys))
            ctx.col_inst = torch.repeat_interleave(torch.arange(len(templates)),
                                                   torch.tensor([t.num_cols for t in templates]))
            ctx.row_inst = torch.repeat_interleave(torch.arange(len(templates)),
                                                   torch.tensor([t.num_rows for t in templates]))
            return torch.tensor(vals, dtype=torch.float64).to(c.device)

        @staticmethod
        def backward(ctx, g):
            g = g.detach().cpu().double()
            return ctx.x * g[ctx.col_inst], ctx.y * g[ctx.row_inst], None, None
except ImportError:  # torch is optional for the C-level API above
    UnrolledLoss = None
    OptimalValue = None

__all__ = ["unrolled", "UnrolledLoss", "OptimalValue", "default_unrolled_opts", "PREC_FP64", "PREC_MIXED",
           "PREC_FP32"]
