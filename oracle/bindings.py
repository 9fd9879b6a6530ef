"""Test infrastructure: ctypes bindings for the oracle libraries.

* ``port()``  -> oracle/_build/liboracle_pdhg.so, the C restatement (oracle/pdhg_oracle.c).
* ``ref()``   -> oracle/_ref/libindus_ref.so, the reference's own CPU code compiled from its
  sources by oracle/Makefile, wrapped by oracle/ref_capi.cpp.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / ``--impl reference`` legs
import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "_build", "liboracle_pdhg.so")
REF_LIB = os.path.join(HERE, "_ref", "libindus_ref.so")

_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_i32p = C.POINTER(C.c_int32)

STATUS_NAMES = {0: "NOT_SOLVED", 1: "OPTIMAL", 2: "INFEASIBLE", 3: "UNBOUNDED",
                4: "INFEASIBLE_OR_UNBOUNDED", 5: "FEASIBLE", 6: "ITERATION_LIMIT",
                7: "TIME_LIMIT", 8: "NODE_LIMIT", 9: "NUMERICAL_ERROR", 10: "MODEL_ERROR",
                11: "UNSUPPORTED"}


class LpStruct(C.Structure):
    """Shared layout of orc_lp / ref_lp / vajra_lp: the reference Model as CSC host arrays."""
    _fields_ = [("num_rows", C.c_int32), ("num_cols", C.c_int32), ("nnz", C.c_int64),
                ("col_ptr", _i64p), ("row_idx", _i32p), ("values", _dp), ("c", _dp),
                ("col_lower", _dp), ("col_upper", _dp), ("row_lower", _dp), ("row_upper", _dp),
                ("sense", C.c_int32), ("objective_offset", C.c_double)]


class OrcOpts(C.Structure):
    _fields_ = [("tolerance", C.c_double), ("gap_tolerance", C.c_double),
                ("time_limit", C.c_double), ("iteration_limit", C.c_int64),
                ("check_frequency", C.c_int32), ("enable_scaling", C.c_int32)]


class OrcResult(C.Structure):
    _fields_ = [("col_value", _dp), ("row_value", _dp), ("row_dual", _dp), ("col_dual", _dp),
                ("status", C.c_int32), ("iterations", C.c_int64), ("objective_value", C.c_double),
                ("restart_count", C.c_int32), ("primal_residual", C.c_double),
                ("dual_residual", C.c_double), ("duality_gap", C.c_double),
                ("spectral_norm_estimate", C.c_double), ("tau", C.c_double), ("sigma", C.c_double),
                ("converged", C.c_int32), ("max_primal_violation", C.c_double),
                ("max_dual_violation", C.c_double), ("is_primal_feasible", C.c_int32),
                ("is_dual_feasible", C.c_int32)]


class DeviceDiagnostics(C.Structure):
    _fields_ = [("primal_residual", C.c_double), ("dual_residual", C.c_double),
                ("objective", C.c_double), ("duality_gap", C.c_double),
                ("converged", C.c_int32), ("numerical_error", C.c_int32)]


class RefOpts(C.Structure):
    _fields_ = [("algorithm", C.c_char_p), ("tolerance", C.c_double), ("gap_tolerance", C.c_double),
                ("time_limit", C.c_double), ("iteration_limit", C.c_int64),
                ("check_frequency", C.c_int32), ("enable_scaling", C.c_int32),
                ("enable_presolve", C.c_int32), ("through_solve", C.c_int32)]


class RefResult(C.Structure):
    _fields_ = [("col_value", _dp), ("row_value", _dp), ("row_dual", _dp), ("col_dual", _dp),
                ("status", C.c_int32), ("iterations", C.c_int64), ("objective_value", C.c_double),
                ("diag_iterations", C.c_int64), ("restart_count", C.c_int32),
                ("primal_residual", C.c_double), ("dual_residual", C.c_double),
                ("duality_gap", C.c_double), ("spectral_norm_estimate", C.c_double),
                ("tau", C.c_double), ("sigma", C.c_double), ("setup_time_sec", C.c_double),
                ("iteration_time_sec", C.c_double), ("total_time_sec", C.c_double),
                ("converged", C.c_int32), ("max_primal_violation", C.c_double),
                ("max_dual_violation", C.c_double), ("is_primal_feasible", C.c_int32),
                ("is_dual_feasible", C.c_int32), ("status_message", C.c_char * 256)]


class RefVerifyOut(C.Structure):
    _fields_ = [("passed", C.c_int32), ("primal_feasible", C.c_int32), ("dual_feasible", C.c_int32),
                ("objective_matches", C.c_int32), ("max_primal_violation", C.c_double),
                ("max_bound_violation", C.c_double), ("max_row_violation", C.c_double),
                ("max_dual_violation", C.c_double), ("max_complementarity_violation", C.c_double),
                ("objective_discrepancy", C.c_double), ("summary", C.c_char * 512)]


def _ptr(a, t):
    return a.ctypes.data_as(t)


class HostLp:
    """Keeps contiguous numpy copies alive and exposes the LpStruct view."""

    def __init__(self, lp):
        self.lp = lp
        self.col_ptr = np.ascontiguousarray(lp.col_ptr, dtype=np.int64)
        self.row_idx = np.ascontiguousarray(lp.row_idx, dtype=np.int32)
        self.values = np.ascontiguousarray(lp.values, dtype=np.float64)
        self.vecs = [np.ascontiguousarray(v, dtype=np.float64) for v in
                     (lp.c, lp.col_lower, lp.col_upper, lp.row_lower, lp.row_upper)]
        self.s = LpStruct(lp.num_rows, lp.num_cols, int(self.col_ptr[-1]),
                          _ptr(self.col_ptr, _i64p), _ptr(self.row_idx, _i32p),
                          _ptr(self.values, _dp), *[_ptr(v, _dp) for v in self.vecs],
                          int(lp.sense), float(lp.objective_offset))


_port = None
_ref = None


def port():
    global _port
    if _port is None:
        if not os.path.exists(PORT_LIB):
            raise FileNotFoundError(f"{PORT_LIB} missing: run `make -C oracle port`")
        lib = C.CDLL(PORT_LIB)
        lib.orc_pdhg_solve.argtypes = [C.POINTER(LpStruct), C.POINTER(OrcOpts), C.POINTER(OrcResult)]
        lib.orc_spectral_norm.restype = C.c_double
        lib.orc_spectral_norm.argtypes = [C.c_int32, C.c_int32, _i64p, _i32p, _dp, C.c_int32, C.c_double]
        lib.orc_ruiz.restype = C.c_int32
        lib.orc_ruiz.argtypes = [C.c_int32, C.c_int32, _i64p, _i32p, _dp, _dp, _dp, _dp, _dp, _dp,
                                 C.c_int32, C.c_double, _dp, _dp]
        lib.orc_device_diagnostics_eval.argtypes = [C.c_int32, C.c_int32] + [_dp] * 9 + [C.POINTER(DeviceDiagnostics)]
        _port = lib
    return _port


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            raise FileNotFoundError(f"{REF_LIB} missing: run `make -C oracle ref` where the reference tree exists")
        lib = C.CDLL(REF_LIB)
        lib.ref_solve.argtypes = [C.POINTER(LpStruct), C.POINTER(RefOpts), C.POINTER(RefResult)]
        lib.ref_spectral_norm.restype = C.c_double
        lib.ref_spectral_norm.argtypes = [C.POINTER(LpStruct), C.c_int32, C.c_double]
        lib.ref_ruiz.argtypes = [C.POINTER(LpStruct), C.c_int32, C.c_double] + [_dp] * 8
        lib.ref_pock_chambolle.argtypes = [C.POINTER(LpStruct), C.c_double, _dp, _dp]
        lib.ref_csc_multiply.argtypes = [C.POINTER(LpStruct), _dp, _dp]
        lib.ref_csc_multiply_transpose.argtypes = [C.POINTER(LpStruct), _dp, _dp]
        lib.ref_verify.argtypes = [C.POINTER(LpStruct), _dp, _dp, C.c_double, C.c_int32, C.c_double,
                                   C.POINTER(RefVerifyOut)]
        _ref = lib
    return _ref


def _alloc_out(lp):
    return {k: np.zeros(n) for k, n in (("x", lp.num_cols), ("row_value", lp.num_rows),
                                          ("y", lp.num_rows), ("d", lp.num_cols))}


def _pack(res_struct, out, names):
    d = {k: getattr(res_struct, k) for k, _ in res_struct._fields_
         if k not in ("col_value", "row_value", "row_dual", "col_dual")}
    if "status_message" in d:
        d["status_message"] = d["status_message"].decode(errors="replace")
    d["status_name"] = STATUS_NAMES.get(d["status"], "?")
    d.update(out)
    return d


def port_solve(lp, tolerance=1e-6, gap_tolerance=1e-6, iteration_limit=1_000_000,
               check_frequency=100, enable_scaling=True):
    """Reference CPU PDHG restated in C (CpuPdhgSolver::solve, pdhg.cpp:70-440)."""
    h = HostLp(lp)
    out = _alloc_out(lp)
    r = OrcResult(_ptr(out["x"], _dp), _ptr(out["row_value"], _dp), _ptr(out["y"], _dp),
                  _ptr(out["d"], _dp))
    o = OrcOpts(tolerance, gap_tolerance, 1e20, iteration_limit, check_frequency, int(enable_scaling))
    rc = port().orc_pdhg_solve(C.byref(h.s), C.byref(o), C.byref(r))
    assert rc == 0
    return _pack(r, out, None)


def ref_solve(lp, tolerance=1e-6, gap_tolerance=1e-6, iteration_limit=1_000_000,
              check_frequency=100, enable_scaling=True, algorithm="pdhg_cpu",
              through_solve=False, enable_presolve=False, time_limit=1e20):
    """The reference's own CPU solver (solve_pdhg_cpu, or indus::solve when through_solve)."""
    h = HostLp(lp)
    out = _alloc_out(lp)
    r = RefResult()
    r.col_value, r.row_value = _ptr(out["x"], _dp), _ptr(out["row_value"], _dp)
    r.row_dual, r.col_dual = _ptr(out["y"], _dp), _ptr(out["d"], _dp)
    o = RefOpts(algorithm.encode(), tolerance, gap_tolerance, time_limit, iteration_limit,
                check_frequency, int(enable_scaling), int(enable_presolve), int(through_solve))
    rc = ref().ref_solve(C.byref(h.s), C.byref(o), C.byref(r))
    if rc != 0:
        raise RuntimeError(r.status_message.decode(errors="replace"))
    return _pack(r, out, None)


def ref_verify(lp, x, row_dual, objective, status, tol=1e-6):
    """indus::verifier::verify_solution (src/engine/verifier.cpp:25-330) on the original model."""
    h = HostLp(lp)
    x = np.ascontiguousarray(x, dtype=np.float64)
    yd = None if row_dual is None else np.ascontiguousarray(row_dual, dtype=np.float64)
    out = RefVerifyOut()
    ref().ref_verify(C.byref(h.s), _ptr(x, _dp), None if yd is None else _ptr(yd, _dp),
                     float(objective), int(status), float(tol), C.byref(out))
    d = {k: getattr(out, k) for k, _ in out._fields_}
    d["summary"] = d["summary"].decode(errors="replace")
    return d


def port_spectral_norm(lp, max_iter=25, tol=1e-4):
    h = HostLp(lp)
    return port().orc_spectral_norm(lp.num_rows, lp.num_cols, _ptr(h.col_ptr, _i64p),
                                    _ptr(h.row_idx, _i32p), _ptr(h.values, _dp), max_iter, tol)


def ref_spectral_norm(lp, max_iter=25, tol=1e-4):
    h = HostLp(lp)
    return ref().ref_spectral_norm(C.byref(h.s), max_iter, tol)


def port_ruiz(lp, max_iters=10, tol=0.05):
    vals = np.array(lp.values, dtype=np.float64)
    vecs = [np.array(v, dtype=np.float64) for v in (lp.c, lp.row_lower, lp.row_upper, lp.col_lower, lp.col_upper)]
    rs, cs = np.zeros(lp.num_rows), np.zeros(lp.num_cols)
    cp = np.ascontiguousarray(lp.col_ptr, dtype=np.int64)
    ri = np.ascontiguousarray(lp.row_idx, dtype=np.int32)
    port().orc_ruiz(lp.num_rows, lp.num_cols, _ptr(cp, _i64p), _ptr(ri, _i32p), _ptr(vals, _dp),
                    *[_ptr(v, _dp) for v in vecs], max_iters, tol, _ptr(rs, _dp), _ptr(cs, _dp))
    return dict(values=vals, c=vecs[0], row_lower=vecs[1], row_upper=vecs[2], col_lower=vecs[3],
                col_upper=vecs[4], row_scale=rs, col_scale=cs)


def ref_ruiz(lp, max_iters=10, tol=0.05):
    h = HostLp(lp)
    vals = np.zeros(lp.nnz)
    c, rl, ru = np.zeros(lp.num_cols), np.zeros(lp.num_rows), np.zeros(lp.num_rows)
    cl, cu = np.zeros(lp.num_cols), np.zeros(lp.num_cols)
    rs, cs = np.zeros(lp.num_rows), np.zeros(lp.num_cols)
    ref().ref_ruiz(C.byref(h.s), max_iters, tol, *[_ptr(a, _dp) for a in (vals, c, rl, ru, cl, cu, rs, cs)])
    return dict(values=vals, c=c, row_lower=rl, row_upper=ru, col_lower=cl, col_upper=cu,
                row_scale=rs, col_scale=cs)


def ref_pock_chambolle(lp, alpha=1.0):
    """The reference's PockChambollePreconditioner::compute (src/linalg/scaling.cpp:179-220) on
    lp's matrix: d_row = 1 / sum_j |a_ij|^(2 - alpha), d_col = 1 / sum_i |a_ij|^alpha."""
    h = HostLp(lp)
    d_row, d_col = np.zeros(lp.num_rows), np.zeros(lp.num_cols)
    ref().ref_pock_chambolle(C.byref(h.s), alpha, _ptr(d_row, _dp), _ptr(d_col, _dp))
    return d_row, d_col


def port_device_diagnostics(ax, rl, ru, aty, c, x, y, cl, cu):
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (ax, rl, ru, aty, c, x, y, cl, cu)]
    out = DeviceDiagnostics()
    port().orc_device_diagnostics_eval(len(ax), len(x), *[_ptr(a, _dp) for a in arrs], C.byref(out))
    return {k: getattr(out, k) for k, _ in out._fields_}
