"""Pins the oracle (oracle/pdhg_oracle.c) before anything is checked against it.

* the reference's own known-answer vectors (tests/golden/kernel_vectors.json), and
* bit-for-bit agreement with the reference's CPU code compiled from its sources
  (oracle/_ref/libindus_ref.so), live where that library exists and through the committed
  fixtures (tests/golden/ref_pdhg_cases.npz) everywhere.
"""
import json
import os

import numpy as np
import pytest

from oracle import bindings as B
from vajra_pdhg import workloads as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KV = json.load(open(os.path.join(GOLDEN, "kernel_vectors.json")))
SCALARS = ("status", "iterations", "objective_value", "restart_count", "primal_residual",
           "dual_residual", "duality_gap", "spectral_norm_estimate", "tau", "sigma",
           "max_primal_violation", "max_dual_violation", "is_primal_feasible", "is_dual_feasible")
needs_ref = pytest.mark.skipif(not B.ref_available(), reason="oracle/_ref not built (no reference tree)")


def lp_from_csr_case(case):
    """Tiny helper LP around a CSR for the orc_* helpers that take a CSC."""
    return case


def test_csr_spmv_golden():
    k = KV["csr_spmv"]
    import ctypes as C
    lib = B.port()
    rp = np.array(k["row_ptr"], np.int64); ci = np.array(k["col_idx"], np.int32)
    v = np.array(k["values"]); x = np.array(k["x"]); y = np.zeros(k["m"])
    lib.orc_csr_multiply(k["m"], B._ptr(rp, B._i64p), B._ptr(ci, B._i32p), B._ptr(v, B._dp), B._ptr(x, B._dp), B._ptr(y, B._dp))
    np.testing.assert_allclose(y, k["expected"], rtol=1e-12, atol=0)


def test_transpose_spmv_golden():
    k = KV["csc_transpose_spmv"]
    lib = B.port()
    cp = np.array(k["col_ptr"], np.int64); ri = np.array(k["row_idx"], np.int32)
    v = np.array(k["values"]); y = np.array(k["y"]); out = np.zeros(k["n"])
    lib.orc_csc_multiply_transpose(k["m"], k["n"], B._ptr(cp, B._i64p), B._ptr(ri, B._i32p), B._ptr(v, B._dp),
                                   B._ptr(y, B._dp), B._ptr(out, B._dp))
    np.testing.assert_array_equal(out, k["expected"])


def test_dual_prox_golden():
    k = KV["dual_prox"]
    lib = B.port()
    ax = np.array(k["ax"]); y = np.array(k["y"]); rl = np.array(k["row_lower"]); ru = np.array(k["row_upper"])
    import ctypes as C
    lib.orc_dual_prox(len(ax), C.c_double(k["sigma"]), B._ptr(ax, B._dp), B._ptr(rl, B._dp), B._ptr(ru, B._dp), B._ptr(y, B._dp))
    np.testing.assert_array_equal(y, k["expected"])


def test_primal_prox_golden():
    k = KV["primal_prox"]
    lib = B.port()
    import ctypes as C
    aty, c = np.array(k["aty"]), np.array(k["c"])
    cl, cu, x = np.array(k["col_lower"]), np.array(k["col_upper"]), np.array(k["x"])
    xb = np.zeros_like(x)
    lib.orc_primal_prox(len(x), C.c_double(k["tau"]), B._ptr(aty, B._dp), B._ptr(c, B._dp), B._ptr(cl, B._dp),
                        B._ptr(cu, B._dp), B._ptr(x, B._dp), B._ptr(xb, B._dp))
    np.testing.assert_array_equal(x, k["expected_x"])
    np.testing.assert_array_equal(xb, k["expected_x_bar"])


def test_diagnostics_golden():
    k = KV["diagnostics"]
    d = B.port_device_diagnostics(k["ax"], k["row_lower"], k["row_upper"], k["aty"], k["c"], k["x"], k["y"],
                                  k["col_lower"], k["col_upper"])
    assert d["primal_residual"] == k["expected_primal_residual"]
    assert d["objective"] == k["expected_objective"]
    assert d["numerical_error"] == k["expected_numerical_error"]


def test_spec_known_answers():
    """tests/test_pdhg.cpp:443-562 known answers through the oracle's formulas."""
    import ctypes as C
    lib = B.port()
    for key in ("spec_csr",):
        k = KV[key]
        rp = np.array(k["row_ptr"], np.int64); ci = np.array(k["col_idx"], np.int32)
        v = np.array(k["values"]); x = np.array(k["x"]); y = np.zeros(len(rp) - 1)
        lib.orc_csr_multiply(len(rp) - 1, B._ptr(rp, B._i64p), B._ptr(ci, B._i32p), B._ptr(v, B._dp), B._ptr(x, B._dp), B._ptr(y, B._dp))
        np.testing.assert_allclose(y, k["expected"], rtol=0, atol=1e-12)
    k = KV["spec_transpose"]
    cp = np.array(k["col_ptr"], np.int64); ri = np.array(k["row_idx"], np.int32)
    v = np.array(k["values"]); y = np.array(k["y"]); out = np.zeros(len(cp) - 1)
    lib.orc_csc_multiply_transpose(len(y), len(cp) - 1, B._ptr(cp, B._i64p), B._ptr(ri, B._i32p), B._ptr(v, B._dp),
                                   B._ptr(y, B._dp), B._ptr(out, B._dp))
    np.testing.assert_allclose(out, k["expected"], atol=1e-12)
    k = KV["spec_dual"]
    for y0, ax, l, u, exp in k["cases"]:
        y = np.array([y0]); a = np.array([ax]); lo = np.array([l]); hi = np.array([u])
        lib.orc_dual_prox(1, C.c_double(k["sigma"]), B._ptr(a, B._dp), B._ptr(lo, B._dp), B._ptr(hi, B._dp), B._ptr(y, B._dp))
        assert abs(y[0] - exp) <= 1e-12
    k = KV["spec_primal"]
    for x0, g, l, u, ex, exb in k["cases"]:
        x = np.array([x0]); v = np.array([g]); c = np.zeros(1); lo = np.array([l]); hi = np.array([u]); xb = np.zeros(1)
        lib.orc_primal_prox(1, C.c_double(k["tau"]), B._ptr(v, B._dp), B._ptr(c, B._dp), B._ptr(lo, B._dp),
                            B._ptr(hi, B._dp), B._ptr(x, B._dp), B._ptr(xb, B._dp))
        assert abs(x[0] - ex) <= 1e-12 and abs(xb[0] - exb) <= 1e-12
    k = KV["spec_residual"]
    d = B.port_device_diagnostics(k["ax"], k["row_lower"], k["row_upper"], [0.0] * 3, k["c"], k["x"], [0.0] * 3,
                                  [-1e20] * 3, [1e20] * 3)
    assert d["primal_residual"] == k["expected_max_violation"]
    assert abs(d["objective"] - k["expected_objective"]) <= 1e-12


def _lp_from_fixture(z, name):
    m, n, iters, sense = (int(v) for v in z[f"{name}/meta"])
    lp = W.LP(m, n, z[f"{name}/col_ptr"], z[f"{name}/row_idx"], z[f"{name}/values"], z[f"{name}/c"],
              z[f"{name}/col_lower"], z[f"{name}/col_upper"], z[f"{name}/row_lower"], z[f"{name}/row_upper"],
              sense=sense)
    return lp, iters


@pytest.mark.parametrize("name", ["eq_20x50", "eq_60x150", "mixed_40x90"])
def test_oracle_matches_reference_fixture(name):
    z = np.load(os.path.join(GOLDEN, "ref_pdhg_cases.npz"))
    lp, iters = _lp_from_fixture(z, name)
    a = B.port_solve(lp, iteration_limit=iters)
    for k in ("x", "y", "d", "row_value"):
        np.testing.assert_array_equal(a[k], z[f"{name}/out_{k}"], err_msg=k)
    s = z[f"{name}/out_scalars"]
    got = [a["status"], a["iterations"], a["objective_value"], a["restart_count"], a["primal_residual"],
           a["dual_residual"], a["duality_gap"], a["spectral_norm_estimate"]]
    np.testing.assert_array_equal(np.array(got, dtype=np.float64), s)


CASES = [("eq", lambda: W.random_planted(30, 70, 3, seed=1), 2000, 100),
         ("eq_cf7", lambda: W.random_planted(50, 120, 5, seed=2), 777, 7),
         ("mixed", lambda: W.small_random(40, 100, 3), 3000, 100),
         ("mixed_noscale", lambda: W.small_random(25, 60, 4), 800, 50)]


@needs_ref
@pytest.mark.parametrize("name,make,iters,cf", CASES)
def test_oracle_bit_identical_to_reference(name, make, iters, cf):
    lp = make()
    scale = not name.endswith("noscale")
    a = B.port_solve(lp, iteration_limit=iters, check_frequency=cf, enable_scaling=scale)
    b = B.ref_solve(lp, iteration_limit=iters, check_frequency=cf, enable_scaling=scale)
    for k in ("x", "y", "d", "row_value"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    for k in SCALARS:
        assert a[k] == b[k], k


@needs_ref
def test_oracle_maximise_and_free_columns():
    lp = W.small_random(30, 60, 9)
    lp.sense = 1
    lp.c = -lp.c
    lp.col_lower = lp.col_lower.copy(); lp.col_upper = lp.col_upper.copy()
    lp.col_lower[::7] = -1e20
    lp.col_upper[::7] = 1e20
    a = B.port_solve(lp, iteration_limit=1500)
    b = B.ref_solve(lp, iteration_limit=1500)
    for k in ("x", "y", "row_value"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    for k in SCALARS:
        assert a[k] == b[k], k


@needs_ref
def test_ruiz_and_norm_bit_identical():
    lp = W.small_random(80, 200, 5)
    a, b = B.port_ruiz(lp), B.ref_ruiz(lp)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert B.port_spectral_norm(lp) == B.ref_spectral_norm(lp)


@needs_ref
def test_reference_runs_the_pdhg_not_simplex():
    """The field-assigned algorithm reaches the reference PDHG (iterations counted)."""
    lp = W.random_planted(20, 50, 3, seed=4)
    r = B.ref_solve(lp, iteration_limit=300, through_solve=True)
    assert r["iterations"] >= 300 or r["status_name"] == "OPTIMAL"
