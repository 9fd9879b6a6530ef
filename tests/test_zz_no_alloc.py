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


def noalloc_call(lib, lp, d, out, stream=None):
    def q(key):
        return p(d[key]) if key in d else None
    return lib.vajra_relative_kkt_noalloc_f64(
        lp.num_rows, lp.num_cols, q("row_ptr"), q("col_idx"), q("csr"), q("col_ptr"), q("row_idx"), q("csc"),
        q("c"), q("cl"), q("cu"), q("rl"), q("ru"), q("x"), q("y"), int(lp.sense), float(lp.objective_offset),
        p(out), stream)


def assert_matches_host(out, lp, x, y, rtol):
    """The device figures against the host FP64 KKT of vajra_pdhg.kkt (different summation order)."""
    from vajra_pdhg.kkt import relative_kkt
    k = relative_kkt(lp, x, y)
    rel_p, rel_d, rel_gap, rel_kkt, pobj, dobj = out.cpu().numpy()
    for got, want in ((rel_p, k["rel_primal"]), (rel_d, k["rel_dual"]), (rel_gap, k["rel_gap"]),
                      (rel_kkt, k["rel_kkt"])):
        assert abs(got - want) <= rtol * (abs(want) + 1e-300) + 1e-15, (got, want)
    assert abs(pobj - k["primal_objective"]) <= rtol * (1 + abs(k["primal_objective"]))
    assert abs(dobj - k["dual_objective"]) <= rtol * (1 + abs(k["dual_objective"]))


def test_noalloc_call_allocates_nothing_and_can_be_captured(cuda):
    """After a first call (which may load the kernels), further calls leave the device's free
    memory unchanged, and a call captured into a CUDA graph -- global capture mode, where an
    allocation or a synchronisation would fail the capture -- replays to the same figures."""
    import torch
    lp = W.small_random(300, 700, 5)
    g = V.solve(lp, precision=V.PREC_FP64)
    d = device_arrays(lp, g["x"], g["y"])
    lib = _capi.lib()
    ref = torch.zeros(6, dtype=torch.float64, device="cuda")
    assert noalloc_call(lib, lp, d, ref) == _capi.OK      # first call on this device
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    outs = [torch.zeros(6, dtype=torch.float64, device="cuda") for _ in range(3)]
    for out in outs[:2]:
        assert noalloc_call(lib, lp, d, out) == _capi.OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        with torch.cuda.graph(graph, stream=side, capture_error_mode="global"):
            st = noalloc_call(lib, lp, d, outs[2], C.c_void_p(side.cuda_stream))
    assert st == _capi.OK, lib.vajra_status_string(st)
    graph.replay()
    torch.cuda.synchronize()
    for out in outs:
        assert torch.equal(out, ref)                        # same kernels, same order: same bits
    del graph


def test_noalloc_lp_without_rows(cuda):
    """An LP with column bounds only (rows = 0): its row-side pointers are NULL."""
    import torch
    n = 50
    rng = np.random.default_rng(11)
    lp = W.LP(0, n, np.zeros(n + 1, np.int64), np.zeros(0, np.int32), np.zeros(0), rng.standard_normal(n),
              np.where(rng.random(n) < 0.8, -rng.random(n), -1e20), np.where(rng.random(n) < 0.8, rng.random(n), 1e20),
              np.zeros(0), np.zeros(0), sense=0, objective_offset=1.25)
    x = np.clip(rng.standard_normal(n), lp.col_lower, lp.col_upper)
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda()
         for k, v in {"col_ptr": lp.col_ptr, "c": lp.c, "cl": lp.col_lower, "cu": lp.col_upper, "x": x}.items()}
    out = torch.zeros(6, dtype=torch.float64, device="cuda")
    st = noalloc_call(_capi.lib(), lp, d, out)
    assert st == _capi.OK
    torch.cuda.synchronize()
    assert_matches_host(out, lp, x, np.zeros(0), 1e-12)


def test_noalloc_at_its_row_limit(cuda):
    """8,388,608 rows, the most the fixed scratch holds (32768 row blocks, the last partial-sum
    slot of the row table written and read), one entry per row; against the host KKT."""
    import torch
    m, n = 8_388_608, 64
    rng = np.random.default_rng(12)
    rows = np.arange(m, dtype=np.int64)
    cols = rows % n
    order = np.lexsort((rows, cols))
    col_ptr = np.zeros(n + 1, np.int64)
    col_ptr[1:] = np.cumsum(np.bincount(cols, minlength=n))
    vals = rng.standard_normal(m)
    eq = rng.random(m) < 0.5
    lo = rng.standard_normal(m)
    lp = W.LP(m, n, col_ptr, rows[order].astype(np.int32), vals[order], rng.standard_normal(n), np.zeros(n),
              np.full(n, 10.0), lo, np.where(eq, lo, lo + rng.random(m)), sense=0, objective_offset=0.0)
    x = rng.random(n) * 10
    y = rng.standard_normal(m)
    d = device_arrays(lp, x, y)
    out = torch.zeros(6, dtype=torch.float64, device="cuda")
    assert noalloc_call(_capi.lib(), lp, d, out) == _capi.OK
    torch.cuda.synchronize()
    assert_matches_host(out, lp, x, y, 1e-9)
    del d
    torch.cuda.empty_cache()
