"""The reference's own test inputs, rebuilt bit-for-bit -- TEST INFRASTRUCTURE.

tests/unit/test_gpu_backend.cpp draws its matrices with std::mt19937 and
libstdc++'s uniform_real_distribution<double>:
  * make_problem(nrows, ncols, density, seed) (:26-49): for every (i, j) in
    row-major order one U(0,1) draw; below `density` it is followed by a
    value draw U(-4, 4); then x = U(-4, 4)^ncols;
  * make_diagonal(n) (:52-65): 2.0 on the diagonal, x = 1.5;
  * the SpMM right-hand sides B = U(lo, hi)^(ncols*k) from their own seeds.
numpy's MT19937 with legacy seeding is std::mt19937(seed); libstdc++'s
generate_canonical<double, 53> takes two 32-bit outputs g1, g2 and returns
(g1 + g2 * 2^32) / 2^64 (clamped below 1); uniform(a, b) = u * (b - a) + a.
"""
from __future__ import annotations

import numpy as np

TWO32 = 4294967296.0
TWO64 = 18446744073709551616.0
ONE_MINUS = np.nextafter(1.0, 0.0)


def _canonical_pairs(seed: int, npairs: int) -> np.ndarray:
    bg = np.random.MT19937()
    bg._legacy_seeding(seed)
    raw = bg.random_raw(2 * npairs).astype(np.float64)
    u = (raw[0::2] + raw[1::2] * TWO32) / TWO64
    return np.where(u >= 1.0, ONE_MINUS, u)


def uniform(seed: int, count: int, lo: float, hi: float) -> np.ndarray:
    return _canonical_pairs(seed, count) * (hi - lo) + lo


def make_problem(nrows: int, ncols: int, density: float, seed: int):
    """Returns (rp, ci, val, x) exactly as make_problem builds them."""
    total = nrows * ncols
    npairs = int(total * (1.0 + density) * 1.05) + 4 * ncols + 1024
    while True:
        u = _canonical_pairs(seed, npairs)
        a = u < density
        k = np.arange(npairs)
        # pair k is a test draw iff it does not directly follow an accepted test
        # draw: T_0 = 1, T_k = 1 - T_{k-1} a_{k-1}. Inside a run of accepted
        # flags T alternates, and it resets to 1 after any rejected flag.
        start = np.where(np.concatenate(([True], ~a[:-1])), k, 0)
        start = np.maximum.accumulate(start)
        is_test = ((k - start) % 2) == 0
        tests = np.flatnonzero(is_test)
        if tests.shape[0] < total + 1:
            npairs *= 2
            continue
        tests = tests[:total]
        acc = a[tests]
        last = tests[-1] if total > 0 else -1
        x_first = last + 1 + (1 if total > 0 and acc[-1] else 0)
        if x_first + ncols > npairs:
            npairs *= 2
            continue
        vals = u[tests[acc] + 1] * 8.0 + (-4.0)
        entry = np.flatnonzero(acc)
        rows = entry // ncols
        cols = entry % ncols
        rp = np.zeros(nrows + 1, dtype=np.int64)
        np.add.at(rp, rows + 1, 1)
        rp = np.cumsum(rp)
        x = u[x_first:x_first + ncols] * 8.0 + (-4.0)
        return rp, cols.astype(np.int64), vals, x


def make_diagonal(n: int):
    rp = np.arange(n + 1, dtype=np.int64)
    ci = np.arange(n, dtype=np.int64)
    return rp, ci, np.full(n, 2.0), np.full(n, 1.5)


def expect_close(got, ref, tol):
    """|got - ref| <= tol * max(1, |ref|) per entry (test_gpu_backend.cpp:67-74)."""
    got, ref = np.asarray(got), np.asarray(ref)
    assert got.shape == ref.shape
    scale = np.maximum(1.0, np.abs(ref))
    bad = np.abs(got - ref) > tol * scale
    assert not bad.any(), f"{bad.sum()} entries off, first at {np.flatnonzero(bad)[:5]}"


def normwise_close(y, y_ref, rp, ci, val, x, tol=1e-12):
    """|y_i - y_ref_i| <= tol * sum_k |a_ik x_k| (+ tiny absolute floor)."""
    m = rp.shape[0] - 1
    rows = np.repeat(np.arange(m), np.diff(rp))
    scale = np.bincount(rows, weights=np.abs(val * x[ci]), minlength=m)
    err = np.abs(np.asarray(y) - np.asarray(y_ref))
    bad = err > tol * scale + 1e-300
    assert not bad.any(), f"{bad.sum()} rows off; worst rel {(err / np.maximum(scale, 1e-300)).max():.3e}"
