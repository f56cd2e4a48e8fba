"""Generates the golden fixtures in this folder from the reference itself.

Run with the reference's source root in REF (oracle/Makefile builds
oracle/_ref/libhnref.so from it): `REF=<dir> python tests/golden/make_golden.py`.
Every output array below is produced by the reference's own code through
oracle/ref_shim.cpp; inputs are rebuilt from their seeds by tests/refcases.py
(the reference tests' mt19937 generators) and the package's lpgen.py.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "indigenous-cpu-gpu-optimization-engine-for-indian-industry_b200"))

import lpgen  # noqa: E402
import oracle as O  # noqa: E402
import refcases as R  # noqa: E402


def dup_zero_case(seed=5, m=50, n=40):
    """Unsorted rows with duplicate columns and explicit zeros."""
    rng = np.random.default_rng(seed)
    rp = np.zeros(m + 1, dtype=np.int64)
    cis, vs = [], []
    for i in range(m):
        k = int(rng.integers(0, 8))
        cis += list(rng.integers(0, n, size=k))
        vs += list(rng.choice([0.0, 1.5, -2.0, 0.25, -1.5], size=k))
        rp[i + 1] = rp[i] + k
    return rp, np.array(cis, dtype=np.int64), np.array(vs, dtype=np.float64), n


def normal_eq_triplets(rp, ci, val, D, reg):
    """The triplet list build_normal_equations emits (interior_point.cpp:144-196)."""
    m = rp.shape[0] - 1
    n = D.shape[0]
    rows = np.repeat(np.arange(m), np.diff(rp))
    order = np.lexsort((rows, ci))  # column-major, rows ascending (the counting sort)
    crow, ccol, cval = rows[order], ci[order], val[order]
    cs = np.searchsorted(ccol, np.arange(n + 1))
    ti, tj, tv = [], [], []
    for j in range(n):
        if D[j] <= 0.0:
            continue
        r, v = crow[cs[j]:cs[j + 1]], cval[cs[j]:cs[j + 1]]
        ti.append(np.repeat(r, r.shape[0]))
        tj.append(np.tile(r, r.shape[0]))
        tv.append(np.outer(v, v).ravel() * D[j])
    ti = np.concatenate(ti) if ti else np.zeros(0, np.int64)
    tj = np.concatenate(tj) if tj else np.zeros(0, np.int64)
    tv = np.concatenate(tv) if tv else np.zeros(0)
    diag = np.zeros(m)
    sel = ti == tj
    for r, v in zip(ti[sel].tolist(), tv[sel].tolist()):
        diag[r] += v
    dyn = max(reg, 1e-12 * max(0.0, diag.max(initial=0.0)))
    ti = np.concatenate([ti, np.arange(m)])
    tj = np.concatenate([tj, np.arange(m)])
    tv = np.concatenate([tv, np.full(m, dyn)])
    return ti, tj, tv, dyn


def main():
    O.build(os.environ.get("REF"))
    assert O.ref() is not None, "reference build missing"
    out = {}
    # CpuBackendTest.SpmvMatchesReference (test_gpu_backend.cpp:90-98) and the
    # CUDA scalar / warp kernel cases (:211-234): y from CPUBackend::spmv
    for name, args in {"spmv_200x150_s42": (200, 150, 0.10, 42),
                       "spmv_1500x1200_s77": (1500, 1200, 0.003, 77),
                       "spmv_300x800_s4242": (300, 800, 0.08, 4242)}.items():
        rp, ci, val, x = R.make_problem(*args)
        out[name + "_y"] = O.ref_backend_spmv(rp, ci, val, x)
    # SpMM cases (:100-124, :260-277): C from CPUBackend::spmm
    for name, (args, k, bseed, lo, hi) in {"spmm_80x60_s7": ((80, 60, 0.2, 7), 4, 99, -2.0, 2.0),
                                          "spmm_400x300_s2024": ((400, 300, 0.05, 2024), 5, 8, -1.0, 1.0)}.items():
        rp, ci, val, _ = R.make_problem(*args)
        B = R.uniform(bseed, args[1] * k, lo, hi)
        out[name + "_C"] = O.ref_backend_spmm(rp, ci, val, B, k, args[1])
    # transpose_multiply and transposed() of the 300x800 case
    rp, ci, val, _ = R.make_problem(300, 800, 0.08, 4242)
    xt = R.uniform(11, 300, -4.0, 4.0)
    out["tmul_300x800_y"] = O.ref_tmultiply(rp, ci, val, xt, 800)
    rpT, ciT, valT = O.ref_transposed(rp, ci, val, 800)
    out["transposed_300x800_rp"], out["transposed_300x800_ci"], out["transposed_300x800_val"] = rpT, ciT, valT
    rp2, ci2, v2, n2 = dup_zero_case()
    out["dupzero_rp"], out["dupzero_ci"], out["dupzero_val"] = rp2, ci2, v2
    a, b, c = O.ref_transposed(rp2, ci2, v2, n2)
    out["dupzero_T_rp"], out["dupzero_T_ci"], out["dupzero_T_val"] = a, b, c
    # normal equations of a scaled 200 x 500 LP (8/col) at a fixed D with zeros,
    # assembled by the reference's from_triplets from the reference's triplets
    lp = lpgen.scaled_problem(lpgen.lp_uniform(200, 500, 8, seed=11))
    D = np.random.default_rng(12).uniform(0.1, 2.0, 500)
    D[::9] = 0.0
    ti, tj, tv, dyn = normal_eq_triplets(lp["rp"], lp["ci"], lp["val"], D, 1e-8)
    nrp, nci, nval = O.ref_from_triplets(200, 200, ti, tj, tv)
    out["ne_D"], out["ne_rp"], out["ne_ci"], out["ne_val"] = D, nrp, nci, nval
    out["ne_dyn"] = np.array([dyn])
    # IPM solves (crossover off) through InteriorPointSolver::solve
    for name, (m, n, k, seed) in {"ipm_60x150": (60, 150, 8, 3), "ipm_200x500": (200, 500, 8, 4)}.items():
        lp = lpgen.lp_uniform(m, n, k, seed)
        r = O.ref_ipm_solve(lp)
        out[name] = np.array([r["status"], r["objective"], r["iterations"]], dtype=np.float64)
        out[name + "_x"] = r["x"]
    path = os.path.join(HERE, "reference_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
