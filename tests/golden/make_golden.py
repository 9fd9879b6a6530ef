"""Regenerates the golden fixtures in this directory.

1. kernel_vectors.json -- the known-answer cases of the reference's own kernel tests,
   transcribed with their file:line:
     tests/test_cuda_kernels.cu:75-107   CSR SpMV with an empty row      -> {-4.5, 0, 14, 11}
     tests/test_cuda_kernels.cu:110-140  CSC transpose SpMV, empty column -> {7, 0, 10}
     tests/test_cuda_kernels.cu:143-173  dual prox ==, <=, >=, ranged      -> {1, 0, -1, 0.5}
     tests/test_cuda_kernels.cu:176-211  primal prox + extrapolation       -> x {0,3,3}, xbar {-1,4,3}
     tests/test_cuda_kernels.cu:214-251  diagnostics: residual 1, objective 8, no NaN
     tests/test_cuda_kernels.cu:254-359  one full iteration (expected values computed by the
                                         oracle, which restates that test's inline CPU loop)
     tests/test_pdhg.cpp:443-562         the CPU "kernel specification" known answers
2. ref_pdhg_cases.npz -- outputs of the reference's own CPU PDHG (compiled from its sources
   by oracle/Makefile into oracle/_ref/libindus_ref.so) on small seeded LPs, so that parity
   can be checked where that library is absent.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "vajra-opt_b200"))

INF = 1e20


def kernel_vectors() -> dict:
    return {
        "csr_spmv": {   # test_cuda_kernels.cu:78-89
            "m": 4, "n": 5, "row_ptr": [0, 2, 2, 5, 6], "col_idx": [0, 2, 0, 3, 4, 1],
            "values": [1.5, -2.0, 3.0, 4.0, -1.0, 5.5], "x": [1.0, 2.0, 3.0, 4.0, 5.0],
            "expected": [-4.5, 0.0, 14.0, 11.0]},
        "csc_transpose_spmv": {   # test_cuda_kernels.cu:113-122
            "n": 3, "m": 4, "col_ptr": [0, 2, 2, 4], "row_idx": [0, 2, 1, 3],
            "values": [1.0, 2.0, -1.0, 3.0], "y": [1.0, 2.0, 3.0, 4.0], "expected": [7.0, 0.0, 10.0]},
        "dual_prox": {   # test_cuda_kernels.cu:145-156
            "sigma": 0.5, "ax": [10.0, 5.0, 2.0, 7.0], "y": [0.0, 0.0, 0.0, 0.0],
            "row_lower": [8.0, -INF, 4.0, 3.0], "row_upper": [8.0, 6.0, INF, 6.0],
            "expected": [1.0, 0.0, -1.0, 0.5]},
        "primal_prox": {   # test_cuda_kernels.cu:178-190
            "tau": 1.0, "aty": [1.0, -2.0, 0.0], "c": [2.0, 1.0, 0.0],
            "col_lower": [0.0, -5.0, -INF], "col_upper": [5.0, 5.0, INF], "x": [1.0, 2.0, 3.0],
            "expected_x": [0.0, 3.0, 3.0], "expected_x_bar": [-1.0, 4.0, 3.0]},
        "diagnostics": {   # test_cuda_kernels.cu:216-249
            "ax": [5.0, 2.0], "row_lower": [0.0, 3.0], "row_upper": [4.0, 10.0], "aty": [0.0, 0.0],
            "c": [2.0, 3.0], "x": [1.0, 2.0], "y": [0.0, 0.0], "col_lower": [0.0, 0.0],
            "col_upper": [10.0, 10.0], "expected_primal_residual": 1.0, "expected_objective": 8.0,
            "expected_numerical_error": 0},
        "full_iteration": {   # test_cuda_kernels.cu:260-277
            "m": 3, "n": 3, "row_ptr": [0, 2, 4, 6], "col_idx": [0, 1, 1, 2, 0, 2],
            "csr_values": [1.0, 2.0, 1.0, -1.0, 2.0, 1.0], "col_ptr": [0, 2, 4, 6],
            "row_idx": [0, 2, 0, 1, 1, 2], "csc_values": [1.0, 2.0, 2.0, 1.0, -1.0, 1.0],
            "row_lower": [4.0, -INF, 3.0], "row_upper": [4.0, 2.0, INF], "c": [1.0, -2.0, 3.0],
            "col_lower": [0.0, -INF, -5.0], "col_upper": [10.0, INF, 5.0],
            "x0": [1.0, 0.0, 1.0], "y0": [0.0, 0.0, 0.0], "sigma": 0.4, "tau": 0.4},
        "spec_csr": {   # test_pdhg.cpp:445-458
            "row_ptr": [0, 2, 2, 5, 6], "col_idx": [0, 2, 0, 1, 2, 1],
            "values": [1.5, -2.0, 3.0, 4.0, -1.0, 5.5], "x": [2.0, 3.0, 4.0],
            "expected": [-5.0, 0.0, 14.0, 16.5]},
        "spec_transpose": {   # test_pdhg.cpp:464-476
            "col_ptr": [0, 2, 2, 4], "row_idx": [0, 2, 1, 2], "values": [1.0, 2.0, -1.0, 3.0],
            "y": [2.0, 4.0, 6.0], "expected": [14.0, 0.0, 14.0]},
        "spec_dual": {   # test_pdhg.cpp:481-496: (y_old, Ax, l, u) -> y_new at sigma 0.5
            "sigma": 0.5, "cases": [[0.0, 10.0, 5.0, 5.0, 2.5], [0.0, 8.0, -INF, 3.0, 2.5],
                                    [0.0, 2.0, 6.0, INF, -2.0], [0.0, 3.0, 2.0, 4.0, 0.0]]},
        "spec_primal": {   # test_pdhg.cpp:501-521: (x_old, grad, l, u) -> (x_new, x_bar) at tau 1
            "tau": 1.0, "cases": [[2.0, 4.0, 0.0, 5.0, 0.0, -2.0], [1.0, -3.0, -INF, INF, 4.0, 7.0],
                                  [8.0, -5.0, -INF, 10.0, 10.0, 12.0]]},
        "spec_residual": {   # test_pdhg.cpp:526-543
            "ax": [10.0, -2.0, 4.0], "row_lower": [0.0, 0.0, 5.0], "row_upper": [8.0, 10.0, 10.0],
            "expected_max_violation": 2.0, "c": [2.0, -1.0, 0.5], "x": [3.0, 4.0, 10.0],
            "expected_objective": 7.0},
    }


def reference_cases() -> dict:
    from oracle import bindings as B
    from vajra_pdhg import workloads as W
    cases = {}
    specs = [("eq_20x50", W.random_planted(20, 50, 3, seed=11), 500),
             ("eq_60x150", W.random_planted(60, 150, 4, seed=12), 1000),
             ("mixed_40x90", W.small_random(40, 90, 13), 1500)]
    for name, lp, iters in specs:
        r = B.ref_solve(lp, iteration_limit=iters)
        for k in ("col_ptr", "row_idx", "values", "c", "col_lower", "col_upper", "row_lower", "row_upper"):
            cases[f"{name}/{k}"] = getattr(lp, k)
        cases[f"{name}/meta"] = np.array([lp.num_rows, lp.num_cols, iters, lp.sense], dtype=np.int64)
        for k in ("x", "y", "d", "row_value"):
            cases[f"{name}/out_{k}"] = r[k]
        cases[f"{name}/out_scalars"] = np.array([r["status"], r["iterations"], r["objective_value"],
                                                 r["restart_count"], r["primal_residual"], r["dual_residual"],
                                                 r["duality_gap"], r["spectral_norm_estimate"]], dtype=np.float64)
    return cases


def main():
    with open(os.path.join(HERE, "kernel_vectors.json"), "w") as f:
        json.dump(kernel_vectors(), f, indent=1)
    np.savez_compressed(os.path.join(HERE, "ref_pdhg_cases.npz"), **reference_cases())
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
