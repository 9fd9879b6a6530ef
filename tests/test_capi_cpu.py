"""C-ABI checks that need no GPU: the library loads, exports every function declared in
include/vajra_pdhg.h, validates its inputs on the host, and refuses to solve without a
device instead of falling back to the CPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import vajra_pdhg as V
from vajra_pdhg import _capi, workloads as W
from conftest import ROOT, cuda_device_present

HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(vajra_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    lib = _capi.lib()
    names = declared_functions()
    assert len(names) >= 17, names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    bound = {s[0] for s in _capi.SIGNATURES}
    assert set(names) <= bound, set(names) - bound


def test_default_opts():
    o = V.default_opts()
    assert o.algorithm == V.ALGO_HALPERN and o.precision == V.PREC_MIXED
    assert o.tolerance == 1e-6 and o.check_frequency == 64 and o.enable_scaling == 1
    assert o.mixed_switch_tolerance == 2e-6 and o.mixed_reflection == 0.8 and o.reflection == 1.0
    assert o.degree_order == 0 and o.spmv_shape_a == 0 and o.spmv_shape_at == 0 and o.autotune == 1
    assert o.restart_sufficient == 0.2 and o.restart_necessary == 0.8 and o.restart_artificial == 0.36
    assert o.handover_mode == -1   # by size: continue the FP32 epoch from 2^20 entries
    with pytest.raises(KeyError):
        V.default_opts(no_such_option=1)


def test_status_strings():
    lib = _capi.lib()
    for s in range(7):
        assert lib.vajra_status_string(s)
    assert lib.vajra_status_string(99) == b"unknown status"


def _lp_struct(lp):
    return V._HostLp(lp)


def test_invalid_inputs_are_rejected_on_the_host():
    lib = _capi.lib()
    lp = W.random_planted(10, 20, 2, seed=0)
    bad = W.LP(**{**lp.__dict__})
    bad.col_ptr = lp.col_ptr.copy()
    bad.col_ptr[3], bad.col_ptr[4] = bad.col_ptr[4] + 1, bad.col_ptr[3]
    h = _lp_struct(bad)
    r = _capi.VajraResult()
    st = lib.vajra_pdhg_solve(C.byref(h.s), None, C.byref(r))
    assert st == _capi.ERR_INVALID_ARGUMENT
    assert r.status == 10 and b"col_ptr" in r.status_message
    crossed = W.LP(**{**lp.__dict__})
    crossed.col_lower = lp.col_lower.copy(); crossed.col_lower[2] = 11.0
    h = _lp_struct(crossed)
    st = lib.vajra_pdhg_solve(C.byref(h.s), None, C.byref(r))
    assert st == _capi.ERR_INVALID_ARGUMENT and b"crossed" in r.status_message
    nanb = W.LP(**{**lp.__dict__})
    nanb.row_upper = lp.row_upper.copy(); nanb.row_upper[1] = np.nan
    h = _lp_struct(nanb)
    assert lib.vajra_pdhg_solve(C.byref(h.s), None, C.byref(r)) == _capi.ERR_INVALID_ARGUMENT
    assert lib.vajra_pdhg_solve(None, None, C.byref(r)) == _capi.ERR_INVALID_ARGUMENT


@pytest.mark.skipif(cuda_device_present(), reason="checks the no-device path")
def test_no_device_means_no_solve():
    """No CPU fallback: without a device the solver reports UNSUPPORTED."""
    lib = _capi.lib()
    lp = W.random_planted(10, 20, 2, seed=0)
    h = _lp_struct(lp)
    r = _capi.VajraResult()
    st = lib.vajra_pdhg_solve(C.byref(h.s), None, C.byref(r))
    assert st == _capi.ERR_NO_DEVICE
    assert r.status == 11
    assert lib.vajra_is_cuda_available() == 0
    info = V.probe_device()
    assert info["available"] == 0 and "None" in info["device_name"]
    with pytest.raises(RuntimeError):
        V.solve(lp)


@pytest.mark.skipif(cuda_device_present(), reason="checks the no-device path")
def test_batch_without_device_and_invalid_instances():
    lps = [W.random_planted(10, 20, 2, seed=s) for s in range(3)]
    with pytest.raises(RuntimeError, match="no CUDA device|vajra_pdhg_solve_batch failed"):
        V.solve_batch(lps)
    bad = W.LP(**{**lps[1].__dict__})
    bad.col_lower = lps[1].col_lower.copy(); bad.col_lower[0] = 20.0
    with pytest.raises(RuntimeError):
        V.solve_batch([lps[0], bad])
