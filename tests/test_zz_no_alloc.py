"""vajra_relative_kkt_noalloc_f64: the FP64 relative-KKT evaluation for callers that cannot
allocate device memory (their device memory belongs to another allocator, or a cudaMalloc
would synchronise a latency-critical loop).  It must report what the allocating solver
entry point reports for the same point.

Collected last (file name) so that a run stopping at the first failure has run every other
test first; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import vajra_pdhg as V
from vajra_pdhg import _capi, workloads as W

pytestmark = pytest.mark.gpu


def device_arrays(lp, x, y):
    """The LP (CSR and CSC of A, c, bounds) and the point, as CUDA tensors kept by the caller."""
    import torch
    A = lp.to_scipy_csc().tocsr()
    A.sort_indices()
    host = {"row_ptr": A.indptr.astype(np.int64), "col_idx": A.indices.astype(np.int32), "csr": A.data,
            "col_ptr": np.asarray(lp.col_ptr, np.int64), "row_idx": np.asarray(lp.row_idx, np.int32),
            "csc": np.asarray(lp.values, float), "c": lp.c, "cl": lp.col_lower, "cu": lp.col_upper,
            "rl": lp.row_lower, "ru": lp.row_upper, "x": x, "y": y}
    return {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in host.items()}


def p(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_kkt_matches_the_solver_on_two_calls_in_a_row(cuda):
    import torch
    maxi = W.small_random(150, 400, 9)
    maxi.sense = 1
    maxi.c = -maxi.c
    maxi.objective_offset = 3.5
    lps = [W.small_random(300, 700, 3), maxi]
    solved = [V.solve(lp, precision=V.PREC_FP64) for lp in lps]     # the allocating entry point
    dev = [device_arrays(lp, g["x"], g["y"]) for lp, g in zip(lps, solved)]
    outs = [torch.zeros(6, dtype=torch.float64, device="cuda") for _ in lps]
    torch.cuda.synchronize()
    lib = _capi.lib()
    for lp, d, out in zip(lps, dev, outs):                          # two calls in a row
        st = lib.vajra_relative_kkt_noalloc_f64(
            lp.num_rows, lp.num_cols, p(d["row_ptr"]), p(d["col_idx"]), p(d["csr"]), p(d["col_ptr"]),
            p(d["row_idx"]), p(d["csc"]), p(d["c"]), p(d["cl"]), p(d["cu"]), p(d["rl"]), p(d["ru"]),
            p(d["x"]), p(d["y"]), int(lp.sense), float(lp.objective_offset), p(out), None)
        assert st == _capi.OK, lib.vajra_status_string(st)
    torch.cuda.synchronize()
    for lp, g, out in zip(lps, solved, outs):
        rel_p, rel_d, rel_gap, rel_kkt, pobj, dobj = out.cpu().numpy()
        # same tolerance as the host-vs-device KKT comparison of tests/test_halpern_gpu.py
        for got, want in ((rel_kkt, g["rel_kkt"]), (rel_p, g["rel_primal"]), (rel_d, g["rel_dual"]),
                          (rel_gap, g["rel_gap"])):
            assert abs(got - want) <= 1e-8 + 1e-3 * want, (got, want)
        obj = -pobj if lp.sense else pobj
        assert abs(obj - g["objective_value"]) <= 1e-9 * (1 + abs(g["objective_value"]))


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    lib = _capi.lib()
    dummy = C.c_void_p(16)   # never dereferenced: the size check comes first
    st = lib.vajra_relative_kkt_noalloc_f64(8_388_609, 10, *([dummy] * 13), 0, 0.0, dummy, None)
    assert st == _capi.ERR_INVALID_ARGUMENT
