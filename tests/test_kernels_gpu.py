"""Kernel-level parity through the C ABI (device pointers): the reference's golden vectors
(tests/test_cuda_kernels.cu:75-359) and bit-identical agreement with the oracle on seeded
random data."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from oracle import bindings as B
from vajra_pdhg import _capi, workloads as W

pytestmark = pytest.mark.gpu
KV = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "kernel_vectors.json")))


_KEEP = []   # device tensors stay referenced until the test module ends


def dev(a, dtype=None):
    """Host array -> CUDA tensor that stays alive (a freed tensor's block would be reused by
    the next allocation while the C call still holds its address)."""
    import torch
    a = np.ascontiguousarray(a if dtype is None else np.asarray(a, dtype=dtype))
    t = torch.from_numpy(a).cuda()
    _KEEP.append(t)
    return t


def p(t):
    assert any(t is k for k in _KEEP), "pass only tensors created by dev()"
    return C.c_void_p(t.data_ptr())


@pytest.fixture(autouse=True)
def _release():
    yield
    import torch
    torch.cuda.synchronize()
    _KEEP.clear()


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def test_csr_spmv_golden(cuda):
    k = KV["csr_spmv"]
    y = dev(np.zeros(k["m"]))
    st = _capi.lib().vajra_csr_spmv_f64(k["m"], p(dev(k["row_ptr"], np.int64)), p(dev(k["col_idx"], np.int32)),
                                        p(dev(k["values"], np.float64)), p(dev(k["x"], np.float64)), p(y), None)
    assert st == 0
    np.testing.assert_allclose(host(y), k["expected"], rtol=1e-12)


def test_csc_transpose_golden(cuda):
    k = KV["csc_transpose_spmv"]
    v = dev(np.zeros(k["n"]))
    st = _capi.lib().vajra_csc_spmv_transpose_f64(k["n"], p(dev(k["col_ptr"], np.int64)), p(dev(k["row_idx"], np.int32)),
                                                  p(dev(k["values"], np.float64)), p(dev(k["y"], np.float64)), p(v), None)
    assert st == 0
    np.testing.assert_allclose(host(v), k["expected"], rtol=1e-12)


def test_dual_and_primal_prox_golden(cuda):
    k = KV["dual_prox"]
    y = dev(k["y"], np.float64)
    assert _capi.lib().vajra_dual_prox_f64(4, k["sigma"], p(dev(k["ax"], np.float64)), p(dev(k["row_lower"], np.float64)),
                                           p(dev(k["row_upper"], np.float64)), p(y), None) == 0
    np.testing.assert_allclose(host(y), k["expected"], rtol=1e-12)
    k = KV["primal_prox"]
    x = dev(k["x"], np.float64)
    xb = dev(np.zeros(3))
    assert _capi.lib().vajra_primal_prox_f64(3, k["tau"], p(dev(k["aty"], np.float64)), p(dev(k["c"], np.float64)),
                                             p(dev(k["col_lower"], np.float64)), p(dev(k["col_upper"], np.float64)),
                                             p(x), p(xb), None) == 0
    np.testing.assert_allclose(host(x), k["expected_x"], rtol=1e-12)
    np.testing.assert_allclose(host(xb), k["expected_x_bar"], rtol=1e-12)


def test_device_diagnostics_golden(cuda):
    k = KV["diagnostics"]
    out = dev(np.zeros(6))   # 48-byte DeviceDiagnostics
    args = [p(dev(k[n], np.float64)) for n in ("ax", "row_lower", "row_upper", "aty", "c", "x", "y", "col_lower", "col_upper")]
    assert _capi.lib().vajra_device_diagnostics_f64(2, 2, *args, p(out), None) == 0
    d = _capi.VajraDeviceDiagnostics.from_buffer_copy(host(out).tobytes())
    assert d.primal_residual == 1.0 and d.objective == 8.0 and d.numerical_error == 0


def test_full_iteration_matches_oracle(cuda):
    k = KV["full_iteration"]
    m, n = k["m"], k["n"]
    x, xb, y = dev(k["x0"], np.float64), dev(k["x0"], np.float64), dev(k["y0"], np.float64)
    w, v = dev(np.zeros(m)), dev(np.zeros(n))
    f = lambda key, dt=np.float64: p(dev(k[key], dt))
    st = _capi.lib().vajra_pdhg_step_f64(m, n, f("row_ptr", np.int64), f("col_idx", np.int32), f("csr_values"),
                                         f("col_ptr", np.int64), f("row_idx", np.int32), f("csc_values"),
                                         f("row_lower"), f("row_upper"), f("c"), f("col_lower"), f("col_upper"),
                                         k["sigma"], k["tau"], p(x), p(xb), p(y), p(w), p(v), None)
    assert st == 0
    # the inline CPU reference of test_cuda_kernels.cu:279-312, through the oracle
    lib = B.port()
    rp = np.array(k["row_ptr"], np.int64); ci = np.array(k["col_idx"], np.int32); cv = np.array(k["csr_values"])
    cp = np.array(k["col_ptr"], np.int64); ri = np.array(k["row_idx"], np.int32); sv = np.array(k["csc_values"])
    hx, hxb, hy = np.array(k["x0"]), np.array(k["x0"]), np.array(k["y0"])
    hw, hv = np.zeros(m), np.zeros(n)
    arr = lambda a: B._ptr(a, B._dp)
    lib.orc_csr_multiply(m, B._ptr(rp, B._i64p), B._ptr(ci, B._i32p), arr(cv), arr(hxb), arr(hw))
    rl, ru = np.array(k["row_lower"]), np.array(k["row_upper"])
    lib.orc_dual_prox(m, C.c_double(k["sigma"]), arr(hw), arr(rl), arr(ru), arr(hy))
    lib.orc_csr_multiply(n, B._ptr(cp, B._i64p), B._ptr(ri, B._i32p), arr(sv), arr(hy), arr(hv))
    c, cl, cu = np.array(k["c"]), np.array(k["col_lower"]), np.array(k["col_upper"])
    lib.orc_primal_prox(n, C.c_double(k["tau"]), arr(hv), arr(c), arr(cl), arr(cu), arr(hx), arr(hxb))
    for got, exp in ((w, hw), (y, hy), (v, hv), (x, hx), (xb, hxb)):
        np.testing.assert_array_equal(host(got), exp)   # tolerance 1e-12 in the reference; bit-exact here


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_spmv_bit_identical_to_oracle_random(cuda, seed):
    lp = W.random_planted(300, 700, 6, seed=seed)
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(lp.num_cols)
    y = rng.standard_normal(lp.num_rows)
    out = dev(np.zeros(lp.num_cols))
    st = _capi.lib().vajra_csc_spmv_transpose_f64(lp.num_cols, p(dev(lp.col_ptr, np.int64)), p(dev(lp.row_idx, np.int32)),
                                                  p(dev(lp.values)), p(dev(y)), p(out), None)
    assert st == 0
    exp = np.zeros(lp.num_cols)
    B.port().orc_csc_multiply_transpose(lp.num_rows, lp.num_cols, B._ptr(np.ascontiguousarray(lp.col_ptr), B._i64p),
                                        B._ptr(np.ascontiguousarray(lp.row_idx), B._i32p),
                                        B._ptr(np.ascontiguousarray(lp.values), B._dp), B._ptr(y, B._dp), B._ptr(exp, B._dp))
    np.testing.assert_array_equal(host(out), exp)
    # f32 form against a float32 torch reference of the same op
    import torch
    out32 = dev(np.zeros(lp.num_cols, np.float32))
    st = _capi.lib().vajra_csc_spmv_transpose_f32(lp.num_cols, p(dev(lp.col_ptr, np.int64)), p(dev(lp.row_idx, np.int32)),
                                                  p(dev(lp.values, np.float32)), p(dev(y, np.float32)), p(out32), None)
    assert st == 0
    A = lp.to_scipy_csc().astype(np.float32)
    ref32 = A.T @ y.astype(np.float32)
    np.testing.assert_allclose(host(out32), ref32, rtol=1e-5, atol=1e-5)


def test_device_diagnostics_many_ctas_match_the_oracle(cuda):
    """1.5M columns and 0.7M rows (a grid of CTAs and the two-stage reduction): maxima exact,
    the objective sum to rounding, against the oracle's sequential evaluation."""
    rng = np.random.default_rng(17)
    m, n = 700_000, 1_500_000
    rl = rng.standard_normal(m); ru = rl + rng.random(m); ru[::7] = 1e20; rl[::5] = -1e20
    ax = rng.standard_normal(m) * 2
    cl = np.where(rng.random(n) < 0.9, 0.0, -1e20); cu = np.where(rng.random(n) < 0.8, 10.0, 1e20)
    x = rng.random(n) * 11 - 0.5
    c, aty, y = rng.standard_normal(n), rng.standard_normal(n), rng.standard_normal(m)
    arrays = (ax, rl, ru, aty, c, x, y, cl, cu)
    keep = [dev(a, np.float64) for a in arrays]
    out = dev(np.zeros(6))
    assert _capi.lib().vajra_device_diagnostics_f64(m, n, *[p(t) for t in keep], p(out), None) == 0
    d = _capi.VajraDeviceDiagnostics.from_buffer_copy(host(out).tobytes())
    o = B.port_device_diagnostics(*arrays)
    assert d.primal_residual == o["primal_residual"] and d.dual_residual == o["dual_residual"]
    assert d.numerical_error == o["numerical_error"] == 0
    assert abs(d.objective - o["objective"]) <= 1e-9 * (1 + abs(o["objective"]))


def test_gather_probe_sums_the_gathered_entries(cuda):
    """vajra_gather_probe_f32: its per-thread partials add up to sum_k x[idx[k]]."""
    rng = np.random.default_rng(21)
    n, count = 300_000, 5_000_003
    x = rng.random(n).astype(np.float32)
    idx = rng.integers(0, n, count).astype(np.int32)
    threads = C.c_int32(0)
    lib = _capi.lib()
    assert lib.vajra_gather_probe_f32(0, None, None, None, C.byref(threads), None) == _capi.ERR_INVALID_ARGUMENT
    assert threads.value > 0
    ti, tx, tp = dev(idx), dev(x), dev(np.zeros(threads.value, np.float32))
    assert lib.vajra_gather_probe_f32(count, p(ti), p(tx), p(tp), C.byref(threads), None) == 0
    want = float(x[idx].astype(np.float64).sum())
    assert abs(float(host(tp).astype(np.float64).sum()) - want) <= 1e-5 * want
