"""vajra_pdhg: Python front end of the B200 restarted-PDHG LP backend (libvajra_pdhg.so).

The solver surface mirrors the reference's PDHG entry points (include/indus/pdhg.hpp,
include/indus/gpu.hpp): ``solve(lp, ...)`` plays ``indus::gpu::solve_pdhg_gpu`` and returns
the Solution fields (col_value, row_value, row_dual, col_dual, status, objective) together
with the PdhgDiagnostics and GpuTimingDiagnostics fields.  All computation happens in the
CUDA library; this module only marshals host arrays through the C ABI.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import ALGO_HALPERN, ALGO_REFERENCE, PREC_FP64, PREC_MIXED

STATUS_NAMES = {0: "NOT_SOLVED", 1: "OPTIMAL", 2: "INFEASIBLE", 3: "UNBOUNDED",
                4: "INFEASIBLE_OR_UNBOUNDED", 5: "FEASIBLE", 6: "ITERATION_LIMIT",
                7: "TIME_LIMIT", 8: "NODE_LIMIT", 9: "NUMERICAL_ERROR", 10: "MODEL_ERROR",
                11: "UNSUPPORTED"}

__all__ = ["solve", "solve_batch", "Solver", "default_opts", "probe_device", "is_cuda_available",
           "last_timing", "scale_lp", "release_cached_memory", "ALGO_REFERENCE", "ALGO_HALPERN", "PREC_FP64", "PREC_MIXED",
           "STATUS_NAMES"]


def _ptr(a, t):
    return a.ctypes.data_as(t)


class _HostLp:
    """Contiguous host copies of an LP (keeps the arrays alive for the C call)."""

    def __init__(self, lp):
        self.col_ptr = np.ascontiguousarray(lp.col_ptr, dtype=np.int64)
        self.row_idx = np.ascontiguousarray(lp.row_idx, dtype=np.int32)
        self.values = np.ascontiguousarray(lp.values, dtype=np.float64)
        self.vecs = [np.ascontiguousarray(v, dtype=np.float64) for v in
                     (lp.c, lp.col_lower, lp.col_upper, lp.row_lower, lp.row_upper)]
        self.s = _capi.VajraLp(int(lp.num_rows), int(lp.num_cols), int(self.col_ptr[-1]),
                               _ptr(self.col_ptr, _capi._i64p), _ptr(self.row_idx, _capi._i32p),
                               _ptr(self.values, _capi._dp), *[_ptr(v, _capi._dp) for v in self.vecs],
                               int(getattr(lp, "sense", 0)), float(getattr(lp, "objective_offset", 0.0)))


def default_opts(**overrides) -> _capi.VajraOpts:
    o = _capi.VajraOpts()
    _capi.lib().vajra_default_opts(C.byref(o))
    for k, v in overrides.items():
        if not hasattr(o, k):
            raise KeyError(f"unknown option {k!r}")
        setattr(o, k, v)
    return o


def _result_dict(r: _capi.VajraResult, out: dict) -> dict:
    d = {k: getattr(r, k) for k, _ in r._fields_ if k not in ("col_value", "row_value", "row_dual", "col_dual")}
    d["status_message"] = d["status_message"].decode(errors="replace")
    d["status_name"] = STATUS_NAMES.get(d["status"], "?")
    d.update(out)
    return d


def _alloc(lp, zeroed=True):
    """Result arrays for one LP.  zeroed=False leaves them uninitialised: for calls that write
    every element (the batched solver copies every instance's whole range before it returns
    OK, and a failed call raises instead of returning them)."""
    m, n = int(lp.num_rows), int(lp.num_cols)
    new = np.zeros if zeroed else np.empty
    out = {"x": new(n), "row_value": new(m), "y": new(m), "d": new(n)}
    r = _capi.VajraResult()
    r.col_value = _ptr(out["x"], _capi._dp)
    r.row_value = _ptr(out["row_value"], _capi._dp)
    r.row_dual = _ptr(out["y"], _capi._dp)
    r.col_dual = _ptr(out["d"], _capi._dp)
    return r, out


def solve(lp, **opts) -> dict:
    """One call: upload, device set-up, iterate, download (vajra_pdhg_solve).

    Returns x (col_value), row_value, y (row_dual, verifier sign convention), d (col_dual)
    and every scalar field of vajra_result.  Raises on a non-OK library status.
    """
    h = _HostLp(lp)
    o = default_opts(**opts)
    r, out = _alloc(lp)
    st = _capi.lib().vajra_pdhg_solve(C.byref(h.s), C.byref(o), C.byref(r))
    res = _result_dict(r, out)
    if st != _capi.OK:
        raise RuntimeError(f"vajra_pdhg_solve failed ({st}): {res['status_message']}")
    return res


def solve_batch(lps, **opts) -> list:
    """Many independent LPs in one call (vajra_pdhg_solve_batch): packed block-diagonally on
    the device, per-instance restarts and termination.  Returns one result dict per LP."""
    hosts = [_HostLp(lp) for lp in lps]
    arr = (_capi.VajraLp * len(lps))(*[h.s for h in hosts])
    res = (_capi.VajraResult * len(lps))()
    outs = []
    for i, lp in enumerate(lps):
        r, out = _alloc(lp, zeroed=False)
        res[i] = r
        outs.append(out)
    o = default_opts(**opts)
    st = _capi.lib().vajra_pdhg_solve_batch(len(lps), arr, C.byref(o), res)
    results = [_result_dict(res[i], outs[i]) for i in range(len(lps))]
    if st != _capi.OK:
        raise RuntimeError(f"vajra_pdhg_solve_batch failed ({st}): {results[0]['status_message']}")
    return results


class Solver:
    """A resident LP (vajra_pdhg_create) that can be solved repeatedly (vajra_pdhg_run)."""

    def __init__(self, lp, **opts):
        self.lp = lp
        self._h = _HostLp(lp)
        self._o = default_opts(**opts)
        self._handle = C.c_void_p()
        _capi.check(_capi.lib().vajra_pdhg_create(C.byref(self._h.s), C.byref(self._o), C.byref(self._handle)),
                    "vajra_pdhg_create")

    def run(self) -> dict:
        r, out = _alloc(self.lp)
        st = _capi.lib().vajra_pdhg_run(self._handle, C.byref(r))
        res = _result_dict(r, out)
        if st != _capi.OK:
            raise RuntimeError(f"vajra_pdhg_run failed ({st}): {res['status_message']}")
        return res

    def close(self):
        if self._handle:
            _capi.lib().vajra_pdhg_destroy(self._handle)
            self._handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def probe_device(device: int = 0) -> dict:
    info = _capi.VajraDeviceInfo()
    st = _capi.lib().vajra_probe_device(device, C.byref(info))
    d = {k: getattr(info, k) for k, _ in info._fields_}
    d["device_name"] = d["device_name"].decode(errors="replace")
    d["status"] = st
    return d


def is_cuda_available() -> bool:
    return bool(_capi.lib().vajra_is_cuda_available())


def last_timing() -> dict:
    t = _capi.VajraTiming()
    _capi.lib().vajra_last_timing(C.byref(t))
    d = {k: getattr(t, k) for k, _ in t._fields_}
    d["device_name"] = d["device_name"].decode(errors="replace")
    d["kernel_mode"] = d["kernel_mode"].decode(errors="replace")
    return d


def scale_lp(lp, **opts) -> dict:
    """The device set-up's scaling of `lp` (vajra_scale_lp): Ruiz, then Pock-Chambolle when
    `pock_chambolle` is on.  Returns the cumulative row / column scales, the scaled values in
    CSC order, the scaled c (negated for maximisation) and the scaled bounds."""
    h = _HostLp(lp)
    o = default_opts(**opts)
    m, n = int(lp.num_rows), int(lp.num_cols)
    out = {"row_scale": np.zeros(m), "col_scale": np.zeros(n), "values": np.zeros(int(h.col_ptr[-1])),
           "c": np.zeros(n), "col_lower": np.zeros(n), "col_upper": np.zeros(n), "row_lower": np.zeros(m),
           "row_upper": np.zeros(m)}
    keys = ("row_scale", "col_scale", "values", "c", "col_lower", "col_upper", "row_lower", "row_upper")
    st = _capi.lib().vajra_scale_lp(C.byref(h.s), C.byref(o), *[C.c_void_p(out[k].ctypes.data) for k in keys])
    _capi.check(st, "vajra_scale_lp")
    return out


def release_cached_memory(device: int = -1) -> int:
    """Return the library's cached device blocks to the driver (vajra_release_cached_memory)."""
    return int(_capi.lib().vajra_release_cached_memory(device))
