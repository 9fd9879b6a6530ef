"""Seeded synthetic LP workloads with the shapes of the benchmark configurations.

Every matrix is returned in canonical CSC form -- rows ascending within a column,
duplicates summed, entries with |v| <= 1e-11 dropped before summation -- which is what the
reference's ``SparseMatrixCSC::set_from_triplets`` produces (src/linalg/sparse.cpp:46-131).
Infinite bounds use the reference's +-1e20 convention (include/indus/model.hpp:16-55).

Workloads (sizes as named in the benchmark configurations; no public dataset is involved):

* ``random_planted``   m equality rows, n columns, k nnz per column at uniform rows,
  N(0,1) values, 0 <= x <= 10.  A planted primal-dual pair (x0, y0) makes x0 optimal:
  40% of x0 at 0, 20% at 10, 40% U(0,10); b = A x0; c = A^T y0 + z with z ~ U(0,1) at the
  lower bound, -U(0,1) at the upper bound, 0 in between.
* ``random_large``     1M x 2M "precision path" LP: 70% equality rows, 30% <= rows with
  slack s0 ~ U(0,1) and y0 = 0 there; column degrees from a truncated power law on
  [2, 2000] whose exponent is solved so that the mean degree is 10 (about 20M nnz);
  values N(0,1) rounded to FP32 so that FP32 storage is exact.
* ``min_cost_flow``    node-arc incidence matrix (+1 tail, -1 head), integer costs
  U{1..100}, capacities U{10..100}, supplies b = A f0 from a random feasible flow.
* ``batch_sizes``      per-instance (m, n, nnz-per-column range) of the batched workload.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

INF = 1e20


@dataclasses.dataclass
class LP:
    """A bounded LP  min/max c^T x  s.t.  row_lower <= A x <= row_upper, col_lower <= x <= col_upper."""

    num_rows: int
    num_cols: int
    col_ptr: np.ndarray      # int64 [n+1]
    row_idx: np.ndarray      # int32 [nnz]
    values: np.ndarray       # float64 [nnz]
    c: np.ndarray
    col_lower: np.ndarray
    col_upper: np.ndarray
    row_lower: np.ndarray
    row_upper: np.ndarray
    sense: int = 0           # 0 minimise, 1 maximise
    objective_offset: float = 0.0
    name: str = ""
    x_planted: np.ndarray | None = None
    y_planted: np.ndarray | None = None      # standard sign convention (reference row_dual)
    planted_objective: float | None = None

    @property
    def nnz(self) -> int:
        return int(self.col_ptr[-1])

    def to_scipy_csc(self):
        import scipy.sparse as sp
        return sp.csc_matrix((self.values, self.row_idx, self.col_ptr),
                             shape=(self.num_rows, self.num_cols))


def canonical_csc(m: int, n: int, rows: np.ndarray, cols: np.ndarray, vals: np.ndarray):
    """Triplets -> canonical CSC (drop |v| <= 1e-11, sort by (col, row), sum duplicates)."""
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    vals = np.asarray(vals, dtype=np.float64)
    keep = ~(np.abs(vals) <= 1e-11)
    rows, cols, vals = rows[keep], cols[keep], vals[keep]
    key = cols * np.int64(m) + rows
    order = np.argsort(key, kind="stable")
    key, vals = key[order], vals[order]
    if key.size:
        first = np.empty(key.size, dtype=bool)
        first[0] = True
        np.not_equal(key[1:], key[:-1], out=first[1:])
        starts = np.flatnonzero(first)
        summed = np.add.reduceat(vals, starts)
        ukey = key[starts]
    else:
        summed = vals
        ukey = key
    ucol = ukey // m
    urow = (ukey - ucol * m).astype(np.int32)
    col_ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(ucol, minlength=n), out=col_ptr[1:])
    return col_ptr, urow, summed.astype(np.float64)


def _csc_matvec(m, col_ptr, row_idx, values, x):
    cols = np.repeat(np.arange(col_ptr.size - 1), np.diff(col_ptr))
    return np.bincount(row_idx, weights=values * x[cols], minlength=m)


def _csc_rmatvec(n, col_ptr, row_idx, values, y):
    cols = np.repeat(np.arange(col_ptr.size - 1), np.diff(col_ptr))
    return np.bincount(cols, weights=values * y[row_idx], minlength=n)


def _planted_x(rng, n, lo=0.0, hi=10.0):
    kind = rng.random(n)
    x0 = rng.uniform(lo, hi, n)
    at_lo = kind < 0.4
    at_hi = (kind >= 0.4) & (kind < 0.6)
    x0[at_lo] = lo
    x0[at_hi] = hi
    return x0, at_lo, at_hi


def random_planted(m: int = 2000, n: int = 5000, nnz_per_col: int | tuple = 8, seed: int = 0,
                   name: str | None = None) -> LP:
    """Equality-constrained random LP with a planted optimum (the 2,000 x 5,000 workload)."""
    rng = np.random.default_rng(seed)
    if isinstance(nnz_per_col, tuple):
        deg = rng.integers(nnz_per_col[0], nnz_per_col[1] + 1, size=n)
    else:
        deg = np.full(n, int(nnz_per_col))
    cols = np.repeat(np.arange(n), deg)
    rows = rng.integers(0, m, size=cols.size)
    vals = rng.standard_normal(cols.size)
    col_ptr, row_idx, values = canonical_csc(m, n, rows, cols, vals)
    x0, at_lo, at_hi = _planted_x(rng, n)
    b = _csc_matvec(m, col_ptr, row_idx, values, x0)
    y0 = rng.standard_normal(m)
    z = np.zeros(n)
    z[at_lo] = rng.uniform(0.0, 1.0, int(at_lo.sum()))
    z[at_hi] = -rng.uniform(0.0, 1.0, int(at_hi.sum()))
    c = _csc_rmatvec(n, col_ptr, row_idx, values, y0) + z
    return LP(m, n, col_ptr, row_idx, values, c, np.zeros(n), np.full(n, 10.0), b.copy(), b.copy(),
              name=name or f"random_planted_{m}x{n}_s{seed}", x_planted=x0, y_planted=y0,
              planted_objective=float(c @ x0))


def power_law_exponent(kmin: int = 2, kmax: int = 2000, mean: float = 10.0) -> float:
    """Exponent a of P(k) ~ k^-a on [kmin, kmax] with the requested mean (bisection)."""
    k = np.arange(kmin, kmax + 1, dtype=np.float64)

    def mean_of(a):
        p = k ** -a
        return float((k * p).sum() / p.sum())

    lo, hi = 1.01, 4.0
    for _ in range(100):
        mid = 0.5 * (lo + hi)
        if mean_of(mid) > mean:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def random_large(m: int = 1_000_000, n: int = 2_000_000, seed: int = 1, eq_frac: float = 0.7,
                 kmin: int = 2, kmax: int = 2000, mean_degree: float = 10.0) -> LP:
    """The 1M x 2M mixed equality / <= LP with heavy-tailed column degrees."""
    rng = np.random.default_rng(seed)
    a = power_law_exponent(kmin, kmax, mean_degree)
    k = np.arange(kmin, kmax + 1)
    p = k.astype(np.float64) ** -a
    cdf = np.cumsum(p / p.sum())
    deg = k[np.minimum(np.searchsorted(cdf, rng.random(n)), k.size - 1)]
    cols = np.repeat(np.arange(n, dtype=np.int64), deg)
    rows = rng.integers(0, m, size=cols.size)
    vals = rng.standard_normal(cols.size).astype(np.float32).astype(np.float64)
    del deg
    col_ptr, row_idx, values = canonical_csc(m, n, rows, cols, vals)
    del rows, cols, vals
    # Summed duplicates may leave FP32-inexact values; round again so FP32 storage is exact.
    values = values.astype(np.float32).astype(np.float64)
    x0, at_lo, at_hi = _planted_x(rng, n)
    ax0 = _csc_matvec(m, col_ptr, row_idx, values, x0)
    is_eq = rng.random(m) < eq_frac
    s0 = rng.uniform(0.0, 1.0, m)
    row_lower = np.where(is_eq, ax0, -INF)
    row_upper = np.where(is_eq, ax0, ax0 + s0)
    y0 = rng.standard_normal(m)
    y0[~is_eq] = 0.0
    z = np.zeros(n)
    z[at_lo] = rng.uniform(0.0, 1.0, int(at_lo.sum()))
    z[at_hi] = -rng.uniform(0.0, 1.0, int(at_hi.sum()))
    c = _csc_rmatvec(n, col_ptr, row_idx, values, y0) + z
    return LP(m, n, col_ptr, row_idx, values, c, np.zeros(n), np.full(n, 10.0), row_lower, row_upper,
              name=f"random_large_{m}x{n}_s{seed}", x_planted=x0, y_planted=y0,
              planted_objective=float(c @ x0))


def min_cost_flow(nodes: int = 200_000, arcs: int = 1_500_000, seed: int = 2) -> LP:
    """Min-cost flow LP on a random graph; feasible by construction, no planted optimum."""
    rng = np.random.default_rng(seed)
    tail = rng.integers(0, nodes, size=arcs)
    head = rng.integers(0, nodes - 1, size=arcs)
    head = head + (head >= tail)                     # uniform over nodes != tail
    cols = np.repeat(np.arange(arcs), 2)
    rows = np.stack([tail, head], axis=1).reshape(-1)
    vals = np.tile(np.array([1.0, -1.0]), arcs)
    col_ptr, row_idx, values = canonical_csc(nodes, arcs, rows, cols, vals)
    cost = rng.integers(1, 101, size=arcs).astype(np.float64)
    cap = rng.integers(10, 101, size=arcs).astype(np.float64)
    f0 = rng.uniform(0.0, 1.0, arcs) * cap
    b = _csc_matvec(nodes, col_ptr, row_idx, values, f0)
    return LP(nodes, arcs, col_ptr, row_idx, values, cost, np.zeros(arcs), cap, b.copy(), b.copy(),
              name=f"min_cost_flow_{nodes}x{arcs}_s{seed}")


def batch_sizes(count: int = 512, seed: int = 3, m_lo: int = 100, m_hi: int = 20_000):
    """(m, n, (kmin, kmax)) per instance of the batched workload: m log-uniform, n = round(U[2,3] m)."""
    rng = np.random.default_rng(seed)
    ms = np.exp(rng.uniform(math.log(m_lo), math.log(m_hi), size=count)).round().astype(int)
    ns = np.round(rng.uniform(2.0, 3.0, size=count) * ms).astype(int)
    return [(int(m), int(n), (4, 12)) for m, n in zip(ms, ns)]


def batch(count: int = 512, seed: int = 3, m_lo: int = 100, m_hi: int = 20_000) -> list[LP]:
    sizes = batch_sizes(count, seed, m_lo, m_hi)
    return [random_planted(m, n, k, seed=seed * 100_003 + i, name=f"batch{i}_{m}x{n}")
            for i, (m, n, k) in enumerate(sizes)]


def small_random(m: int, n: int, seed: int, density_per_col: int = 3, kinds: bool = True) -> LP:
    """Small mixed-sense LP (==, <=, >=, ranged rows; boxed, one-sided and free columns)."""
    rng = np.random.default_rng(seed)
    base = random_planted(m, n, min(density_per_col, m), seed=seed)
    if not kinds:
        return base
    ax0 = _csc_matvec(m, base.col_ptr, base.row_idx, base.values, base.x_planted)
    kind = rng.integers(0, 4, size=m)
    rl = ax0.copy()
    ru = ax0.copy()
    slack = rng.uniform(0.1, 1.0, m)
    rl[kind == 1] = -INF
    ru[kind == 1] = ax0[kind == 1] + slack[kind == 1]
    rl[kind == 2] = ax0[kind == 2] - slack[kind == 2]
    ru[kind == 2] = INF
    rl[kind == 3] = ax0[kind == 3] - slack[kind == 3]
    ru[kind == 3] = ax0[kind == 3] + slack[kind == 3]
    base.row_lower, base.row_upper = rl, ru
    base.y_planted = None
    base.planted_objective = None
    base.name = f"small_random_{m}x{n}_s{seed}"
    return base
