"""Seeded synthetic LP generators for the workloads this library is measured on.

Every instance is a feasible, bounded LP in the reference's standard shape
    min c^T x  s.t.  A x = b,  x >= 0
built as: per column j, c_j distinct uniform rows; values sign * U(0.1, 1);
x0 ~ U(0.5, 2)^n, b = A x0; y0 ~ N(0, 1)^m, s0 ~ U(0.5, 2)^n, c = A^T y0 + s0
(x0 and (y0, s0) are a strictly feasible primal / dual pair, so an optimum
exists). Column-count laws:
  * lp_uniform(m, n, k): k nonzeros per column (the m=2000, n=5000, 8/col LP;
    the 4096-instance batch with 6/col; the branch-and-bound base LP).
  * zipf_counts(n): truncated Zipf(1.5) on [1, 2000] by an inverse-CDF table,
    optionally rescaled to a target nnz (the m=200k, n=500k LP at ~5.2M nnz).
Seeds are numpy PCG64 seeds; the same seed gives the same LP everywhere.
CSR rows are sorted by column, entries distinct: the layout SparseMatrix::
from_triplets produces (core/numerical/sparse_matrix.cpp:8-53).
"""
from __future__ import annotations

import math

import numpy as np


def zipf_counts(n: int, rng: np.random.Generator, s: float = 1.5, cmax: int = 2000,
                target_nnz: int | None = None) -> np.ndarray:
    k = np.arange(1, cmax + 1, dtype=np.float64)
    w = k ** (-s)
    cdf = np.cumsum(w) / w.sum()
    u = rng.random(n)
    c = np.searchsorted(cdf, u, side="right") + 1
    c = np.minimum(c, cmax).astype(np.int64)
    if target_nnz is not None:
        c = np.maximum(1, np.rint(c * (target_nnz / c.sum()))).astype(np.int64)
    return c


def _distinct_rows(m: int, counts: np.ndarray, rng: np.random.Generator):
    """For each column j draw counts[j] distinct rows in [0, m). Returns
    (cols, rows) sorted by (col, row)."""
    n = counts.shape[0]
    if np.any(counts > m):
        raise ValueError("column count exceeds m")
    cols = np.repeat(np.arange(n, dtype=np.int64), counts)
    rows = rng.integers(0, m, size=cols.shape[0], dtype=np.int64)
    for _ in range(1000):
        key = cols * m + rows
        order = np.argsort(key, kind="stable")
        ks = key[order]
        dup = np.zeros(ks.shape[0], dtype=bool)
        dup[1:] = ks[1:] == ks[:-1]
        if not dup.any():
            return ks // m, ks % m
        bad = order[dup]
        rows[bad] = rng.integers(0, m, size=bad.shape[0], dtype=np.int64)
    raise RuntimeError("could not draw distinct rows")


def _csr_from_cols(m: int, n: int, cols: np.ndarray, rows: np.ndarray, vals: np.ndarray):
    order = np.lexsort((cols, rows))
    r, c, v = rows[order], cols[order], vals[order]
    rp = np.zeros(m + 1, dtype=np.int64)
    np.add.at(rp, r + 1, 1)
    np.cumsum(rp, out=rp)
    return rp, c.astype(np.int64), v


def csr_matvec(rp, ci, val, x):
    m = rp.shape[0] - 1
    rows = np.repeat(np.arange(m), np.diff(rp))
    return np.bincount(rows, weights=val * x[ci], minlength=m)


def csr_tmatvec(rp, ci, val, y, n):
    m = rp.shape[0] - 1
    rows = np.repeat(np.arange(m), np.diff(rp))
    return np.bincount(ci, weights=val * y[rows], minlength=n)


def lp_from_counts(m: int, counts: np.ndarray, seed: int) -> dict:
    rng = np.random.default_rng(seed)
    n = counts.shape[0]
    cols, rows = _distinct_rows(m, counts, rng)
    sign = np.where(rng.random(cols.shape[0]) < 0.5, -1.0, 1.0)
    vals = sign * rng.uniform(0.1, 1.0, size=cols.shape[0])
    rp, ci, val = _csr_from_cols(m, n, cols, rows, vals)
    x0 = rng.uniform(0.5, 2.0, size=n)
    y0 = rng.standard_normal(m)
    s0 = rng.uniform(0.5, 2.0, size=n)
    b = csr_matvec(rp, ci, val, x0)
    c = csr_tmatvec(rp, ci, val, y0, n) + s0
    return {"m": m, "n": n, "rp": rp, "ci": ci, "val": val, "b": b, "c": c,
            "x0": x0, "y0": y0, "s0": s0, "seed": seed}


def lp_uniform(m: int, n: int, k: int, seed: int) -> dict:
    """k distinct nonzeros per column (e.g. m=2000, n=5000, k=8)."""
    return lp_from_counts(m, np.full(n, k, dtype=np.int64), seed)


def lp_staircase(periods: int, k: int, seed: int) -> dict:
    """A multi-period (staircase) LP: `periods` blocks of k EQ rows, 2k
    columns per block, each column with 4 distinct rows in its own block and
    2 in the next; values and feasibility as lp_from_counts (b = A x0,
    c = A^T y0 + s0). Its normal matrix is block tridiagonal, so a
    fill-reducing ordering keeps the factor sparse."""
    rng = np.random.default_rng(seed)
    m, n = periods * k, periods * 2 * k
    rows, cols = [], []
    for j in range(n):
        t = j // (2 * k)
        own = rng.choice(k, 4, replace=False) + t * k
        nxt = rng.choice(k, 2, replace=False) + (t + 1) * k if t + 1 < periods else np.zeros(0, dtype=np.int64)
        r = np.concatenate([own, nxt])
        rows.append(r)
        cols.append(np.full(r.shape[0], j))
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    sign = np.where(rng.random(cols.shape[0]) < 0.5, -1.0, 1.0)
    vals = sign * rng.uniform(0.1, 1.0, size=cols.shape[0])
    rp, ci, val = _csr_from_cols(m, n, cols, rows, vals)
    x0 = rng.uniform(0.5, 2.0, size=n)
    y0 = rng.standard_normal(m)
    s0 = rng.uniform(0.5, 2.0, size=n)
    return {"m": m, "n": n, "rp": rp, "ci": ci, "val": val, "b": csr_matvec(rp, ci, val, x0),
            "c": csr_tmatvec(rp, ci, val, y0, n) + s0, "x0": x0, "y0": y0, "s0": s0, "seed": seed}


def lp_zipf(m: int = 200_000, n: int = 500_000, seed: int = 1000, target_nnz: int | None = 5_000_000) -> dict:
    """Large LP with Zipf(1.5) column counts clipped to [1, 2000]; with
    target_nnz the counts are rescaled (c_j <- max(1, round(c_j * t / sum c)))."""
    rng = np.random.default_rng(seed + 7919)
    counts = zipf_counts(n, rng, target_nnz=target_nnz)
    counts = np.minimum(counts, m)
    return lp_from_counts(m, counts, seed)


def batch_sizes(count: int = 4096, lo: int = 50, hi: int = 2000, seed: int = 2000) -> np.ndarray:
    """m log-uniform in [lo, hi] for the batched configuration."""
    rng = np.random.default_rng(seed)
    return np.rint(np.exp(rng.uniform(math.log(lo), math.log(hi), size=count))).astype(np.int64)


def scaled_problem(lp: dict) -> dict:
    """The problem HyperNova's IPM actually iterates on for an all-EQ,
    x >= 0 LP: rows scaled by 1/max|a_ij|, then columns by 1/max|col|
    (build_standard_form, core/lp/interior_point.cpp:282-371)."""
    rp, ci, val = lp["rp"], lp["ci"], lp["val"]
    m, n = lp["m"], lp["n"]
    rows = np.repeat(np.arange(m), np.diff(rp))
    rowmax = np.zeros(m)
    np.maximum.at(rowmax, rows, np.abs(val))
    gamma = np.where(rowmax > 0, 1.0 / np.where(rowmax > 0, rowmax, 1.0), 1.0)
    v1 = gamma[rows] * val
    colmax = np.zeros(n)
    np.maximum.at(colmax, ci, np.abs(v1))
    cs = np.where(colmax > 0, 1.0 / np.where(colmax > 0, colmax, 1.0), 1.0)
    v2 = v1 * cs[ci]
    return {"m": m, "n": n, "rp": rp, "ci": ci, "val": v2, "b": gamma * lp["b"], "c": lp["c"] * cs,
            "col_scale": cs, "row_scale": gamma}


def bb_nodes(base: dict, count: int = 2048, kmax: int = 40, seed: int = 3000):
    """Branch-and-bound style node relaxations of `base` (x >= 0 LP): each
    node picks k ~ U{1..kmax} distinct variables, perturbs x0_j by
    U(-0.5, 0.5) and sets ub = floor(.) or lb = ceil(.) (coin flip, clipped
    to >= 0). Returns a list of (lb, ub) arrays."""
    rng = np.random.default_rng(seed)
    n = base["n"]
    nodes = []
    for _ in range(count):
        k = int(rng.integers(1, kmax + 1))
        js = rng.choice(n, size=k, replace=False)
        v = base["x0"][js] + rng.uniform(-0.5, 0.5, size=k)
        lb = np.zeros(n)
        ub = np.full(n, np.inf)
        up = rng.random(k) < 0.5
        ub[js[up]] = np.maximum(np.floor(v[up]), 0.0)
        lb[js[~up]] = np.maximum(np.ceil(v[~up]), 0.0)
        nodes.append((lb, ub))
    return nodes
