"""CPU: the oracle (C restatement) pinned against the reference.

Three pins: known-answer tests of the reference's own unit tests
(tests/unit/test_numerical.cpp:11-87), golden fixtures produced by the
reference's code (tests/golden/reference_golden.npz, made by
tests/golden/make_golden.py), and -- where oracle/_ref was built from the
reference sources -- direct comparison with the compiled reference.
"""
import os

import numpy as np
import pytest

import lpgen
import oracle as O
import refcases as R

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_golden.npz"))


def csr(triplets, m):
    t = sorted(triplets)
    rp = np.zeros(m + 1, dtype=np.int64)
    for r, _, _ in t:
        rp[r + 1] += 1
    return np.cumsum(rp), np.array([c for _, c, _ in t], dtype=np.int64), np.array([v for *_, v in t])


def test_known_answer_multiply():
    # SparseMatrixTest.MatrixVectorMultiply (test_numerical.cpp:33-46)
    rp, ci, val = csr([(0, 0, 1.0), (0, 1, 2.0), (1, 0, 3.0), (1, 2, 4.0), (2, 1, 5.0), (2, 2, 6.0)], 3)
    y = O.multiply(rp, ci, val, np.array([1.0, 2.0, 3.0]))
    assert y.tolist() == [1.0 * 1.0 + 2.0 * 2.0, 3.0 * 1.0 + 4.0 * 3.0, 5.0 * 2.0 + 6.0 * 3.0]


def test_known_answer_transpose():
    # SparseMatrixTest.Transpose (test_numerical.cpp:48-64)
    rp, ci, val = csr([(0, 0, 1.0), (0, 1, 2.0), (1, 0, 3.0), (1, 2, 4.0)], 2)
    rpT, ciT, valT = O.transposed(rp, ci, val, 3)
    dense = np.zeros((3, 2))
    for i in range(3):
        for k in range(rpT[i], rpT[i + 1]):
            dense[i, ciT[k]] = valT[k]
    assert dense.tolist() == [[1.0, 3.0], [2.0, 0.0], [0.0, 4.0]]


def test_known_answer_sum_duplicates():
    # SparseMatrixTest.SumDuplicates (test_numerical.cpp:66-76), through transposed()
    rp = np.array([0, 2, 3]); ci = np.array([0, 0, 1]); val = np.array([1.0, 2.0, 3.0])
    rpT, ciT, valT = O.transposed(rp, ci, val, 2)
    assert rpT.tolist() == [0, 1, 2] and ciT.tolist() == [0, 1] and valT.tolist() == [3.0, 3.0]


@pytest.mark.parametrize("name,args", [("spmv_200x150_s42", (200, 150, 0.10, 42)),
                                       ("spmv_1500x1200_s77", (1500, 1200, 0.003, 77)),
                                       ("spmv_300x800_s4242", (300, 800, 0.08, 4242))])
def test_port_spmv_matches_golden(name, args):
    rp, ci, val, x = R.make_problem(*args)
    assert np.array_equal(O.multiply(rp, ci, val, x), GOLD[name + "_y"])


@pytest.mark.parametrize("name,args,k,bseed,lo,hi", [
    ("spmm_80x60_s7", (80, 60, 0.2, 7), 4, 99, -2.0, 2.0),
    ("spmm_400x300_s2024", (400, 300, 0.05, 2024), 5, 8, -1.0, 1.0)])
def test_port_spmm_matches_golden(name, args, k, bseed, lo, hi):
    rp, ci, val, _ = R.make_problem(*args)
    B = R.uniform(bseed, args[1] * k, lo, hi)
    assert np.array_equal(O.spmm(rp, ci, val, B, k), GOLD[name + "_C"])


def test_port_transpose_multiply_matches_golden():
    rp, ci, val, _ = R.make_problem(300, 800, 0.08, 4242)
    xt = R.uniform(11, 300, -4.0, 4.0)
    assert np.array_equal(O.tmultiply(rp, ci, val, xt, 800), GOLD["tmul_300x800_y"])
    # the IPM's matvec_t is the same scatter without the x_i == 0 skip
    assert np.array_equal(O.matvec_t(rp, ci, val, xt, 800), GOLD["tmul_300x800_y"])


def test_port_transposed_matches_golden():
    rp, ci, val, _ = R.make_problem(300, 800, 0.08, 4242)
    rpT, ciT, valT = O.transposed(rp, ci, val, 800)
    assert np.array_equal(rpT, GOLD["transposed_300x800_rp"].astype(np.int64))
    assert np.array_equal(ciT, GOLD["transposed_300x800_ci"].astype(np.int64))
    assert np.array_equal(valT, GOLD["transposed_300x800_val"])


def test_port_transposed_duplicates_and_zeros_match_golden():
    rpT, ciT, valT = O.transposed(GOLD["dupzero_rp"], GOLD["dupzero_ci"], GOLD["dupzero_val"], 40)
    assert np.array_equal(rpT, GOLD["dupzero_T_rp"].astype(np.int64))
    assert np.array_equal(ciT, GOLD["dupzero_T_ci"].astype(np.int64))
    assert np.array_equal(valT, GOLD["dupzero_T_val"])
    assert len(ciT) < len(GOLD["dupzero_ci"])  # the case does merge and drop


def test_port_normal_equations_match_golden():
    lp = lpgen.scaled_problem(lpgen.lp_uniform(200, 500, 8, seed=11))
    D = GOLD["ne_D"]
    rpN, ciN, vN, dyn = O.normal_equations(lp["rp"], lp["ci"], lp["val"], D, 1e-8, 500)
    assert np.array_equal(rpN, GOLD["ne_rp"].astype(np.int64))
    assert np.array_equal(ciN, GOLD["ne_ci"].astype(np.int64))
    assert dyn == GOLD["ne_dyn"][0]
    # duplicate sums: the reference's std::sort leaves their order open
    _, _, absN, _ = O.normal_equations(lp["rp"], lp["ci"], np.abs(lp["val"]), D, 0.0, 500)
    assert np.all(np.abs(vN - GOLD["ne_val"]) <= 1e-12 * (absN + dyn))


def test_port_pattern_is_structural_pattern():
    lp = lpgen.lp_uniform(200, 500, 8, seed=11)
    D = np.ones(500)
    rpN, ciN, _, _ = O.normal_equations(lp["rp"], lp["ci"], lp["val"], D, 1e-8, 500)
    rpP, ciP = O.ada_pattern(lp["rp"], lp["ci"], 500)
    assert np.array_equal(rpN, rpP) and np.array_equal(ciN, ciP.astype(np.int64))


def test_port_small_vector_ops():
    rng = np.random.default_rng(0)
    a, b = rng.standard_normal(1000), rng.standard_normal(1000)
    s = 0.0
    for u, v in zip(a.tolist(), b.tolist()):
        s += u * v
    assert O.dot(a, b) == s
    v = a.copy(); v[3] = np.nan
    assert O.norm_inf(v) == np.max(np.abs(np.delete(a, 3)))
    assert np.array_equal(O.axpy(0.5, a, b), b + 0.5 * a)
    d = b.copy()
    assert O.max_step(np.abs(a) + 1, d) == min(1.0, 0.99 * np.min(-(np.abs(a) + 1)[d < 0] / d[d < 0]))


def test_merge_tiles_cover_path():
    rp, ci, _, _ = R.make_problem(300, 800, 0.08, 4242)
    rp32 = rp.astype(np.int32)
    nnz, m, items = int(rp[-1]), 300, 2048
    nt = (m + nnz + items - 1) // items
    row, nz = O.merge_tiles(rp32, nnz, items, nt)
    assert row[0] == 0 and nz[0] == 0 and row[-1] == m and nz[-1] == nnz
    assert np.all(np.diff(row.astype(np.int64) + nz) <= items)
    # every coordinate lies on the merge path: rp[row] <= nz <= rp[row+1]
    assert np.all(rp32[row[:-1]] <= nz[:-1]) and np.all(nz[:-1] <= rp32[np.minimum(row[:-1] + 1, m)])


needs_ref = pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built (needs the reference sources)")


@needs_ref
def test_port_matches_compiled_reference_random():
    lp = lpgen.lp_uniform(300, 700, 8, seed=21)
    rp, ci, val = lp["rp"], lp["ci"], lp["val"]
    x = np.random.default_rng(1).standard_normal(700)
    assert np.array_equal(O.multiply(rp, ci, val, x), O.ref_multiply(rp, ci, val, x))
    xt = np.random.default_rng(2).standard_normal(300)
    assert np.array_equal(O.tmultiply(rp, ci, val, xt, 700), O.ref_tmultiply(rp, ci, val, xt, 700))
    for a, b in zip(O.transposed(rp, ci, val, 700), O.ref_transposed(rp, ci, val, 700)):
        assert np.array_equal(np.asarray(a, np.float64), np.asarray(b, np.float64))


@needs_ref
def test_reference_ipm_known_answers():
    # InteriorPointTest.WarmStartCrossoverProducesExactCertificate (test_lp.cpp:347-377):
    # max x1 + 2 x2, x1 + x2 <= 10, x1 <= 5, 0 <= x <= 10 -> objective 20
    lp = {"m": 2, "n": 2, "rp": np.array([0, 2, 3]), "ci": np.array([0, 1, 0]),
          "val": np.array([1.0, 1.0, 1.0]), "b": np.array([10.0, 5.0]), "c": np.array([1.0, 2.0])}
    r = O.ref_ipm_solve(lp, sense=np.array([0, 0]), ub=np.array([10.0, 10.0]), maximize=True, crossover=True)
    assert r["status"] == 1 and abs(r["objective"] - 20.0) < 1e-6
    # IterationLimitReportsIncumbent (:306-325): ITER_LIMIT (6) with an incumbent
    r = O.ref_ipm_solve(lp, sense=np.array([0, 0]), ub=np.array([10.0, 10.0]), maximize=True, max_iter=1)
    assert r["status"] == 6 and r["objective"] != 0.0


@needs_ref
@pytest.mark.parametrize("name,args", [("ipm_60x150", (60, 150, 8, 3)), ("ipm_200x500", (200, 500, 8, 4))])
def test_reference_ipm_reproduces_golden(name, args):
    r = O.ref_ipm_solve(lpgen.lp_uniform(*args))
    g = GOLD[name]
    assert r["status"] == int(g[0]) and r["objective"] == g[1] and r["iterations"] == int(g[2])


@needs_ref
def test_port_normal_equations_match_reference_function():
    # the reference's own build_normal_equations, reached by ref_ipm_shim.cpp
    lp = lpgen.scaled_problem(lpgen.lp_uniform(300, 750, 8, seed=5))
    D = np.random.default_rng(6).uniform(0.01, 100.0, 750)
    D[::11] = 0.0
    rpR, ciR, vR = O.ref_normal_equations(lp["rp"], lp["ci"], lp["val"], D, 1e-8, 750)
    rpP, ciP, vP, dyn = O.normal_equations(lp["rp"], lp["ci"], lp["val"], D, 1e-8, 750)
    assert np.array_equal(rpR.astype(np.int64), rpP) and np.array_equal(ciR.astype(np.int64), ciP)
    _, _, absN, _ = O.normal_equations(lp["rp"], lp["ci"], np.abs(lp["val"]), D, 0.0, 750)
    assert np.all(np.abs(vR - vP) <= 1e-12 * (absN + dyn))


@needs_ref
def test_port_matvec_t_and_max_step_match_reference_functions():
    lp = lpgen.lp_uniform(300, 750, 8, seed=5)
    x = np.random.default_rng(7).standard_normal(300)
    assert np.array_equal(O.matvec_t(lp["rp"], lp["ci"], lp["val"], x, 750),
                          O.ref_matvec_t(lp["rp"], lp["ci"], lp["val"], x, 750))
    rng = np.random.default_rng(8)
    v, d = rng.uniform(0.1, 2, 1000), rng.standard_normal(1000)
    assert O.max_step(v, d) == O.ref_max_step(v, d)
    assert O.max_step(v, np.abs(d)) == O.ref_max_step(v, np.abs(d)) == 0.99  # 0.99 * 1 when nothing blocks


def test_port_normal_rows_equal_full_restatement():
    """The row-restricted restatement (used at sizes whose triplet list does
    not fit) gives the full restatement's rows bit for bit, including dyn_reg
    taken over all rows and repeated / unordered row requests."""
    lp = lpgen.scaled_problem(lpgen.lp_uniform(300, 750, 8, 3))
    D = np.random.default_rng(1).uniform(0.1, 10, 750)
    D[::13] = 0.0
    rpN, ciN, vN, dyn = O.normal_equations(lp["rp"], lp["ci"], lp["val"], D, 1e-8, 750)
    rows = np.array([5, 0, 299, 17, 17, 150])
    rpS, ciS, vS, aS, dynS = O.normal_rows(lp["rp"], lp["ci"], lp["val"], D, 1e-8, 750, rows)
    assert dynS == dyn
    for s, i in enumerate(rows):
        a, b, c, d = rpN[i], rpN[i + 1], rpS[s], rpS[s + 1]
        assert np.array_equal(ciN[a:b], ciS[c:d]) and np.array_equal(vN[a:b], vS[c:d])
        assert np.all(aS[c:d] >= np.abs(vS[c:d]))
