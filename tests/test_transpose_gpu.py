"""GPU: integer work is bit-exact -- device A^T against SparseMatrix::transposed
(golden fixtures from the reference + the oracle), merge-path tile tables
against the oracle's restatement, and transpose(transpose(A)) == A at the
full 200k x 500k size."""
import os

import numpy as np
import pytest

import lpgen
import oracle as O
import refcases as R

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_golden.npz"))


def assert_transpose_equal(A, ref):
    rpT, ciT, valT = A.export(trans=1)
    assert np.array_equal(rpT.astype(np.int64), np.asarray(ref[0]).astype(np.int64))
    assert np.array_equal(ciT.astype(np.int64), np.asarray(ref[1]).astype(np.int64))
    assert np.array_equal(valT, np.asarray(ref[2]))  # same doubles, same bits


def test_transpose_matches_reference_golden(hn):
    rp, ci, val, _ = R.make_problem(300, 800, 0.08, 4242)
    A = hn.Csr(300, 800, rp, ci, val)
    assert_transpose_equal(A, (GOLD["transposed_300x800_rp"], GOLD["transposed_300x800_ci"],
                               GOLD["transposed_300x800_val"]))


def test_transpose_duplicates_zeros_match_reference_golden(hn):
    A = hn.Csr(50, 40, GOLD["dupzero_rp"], GOLD["dupzero_ci"], GOLD["dupzero_val"])
    assert_transpose_equal(A, (GOLD["dupzero_T_rp"], GOLD["dupzero_T_ci"], GOLD["dupzero_T_val"]))
    assert A.nnz_t < A.nnz


@pytest.mark.parametrize("args", [(200, 150, 0.10, 42), (1500, 1200, 0.003, 77), (4000, 3000, 0.08, 31337)])
def test_transpose_reference_cases(hn, args):
    rp, ci, val, _ = R.make_problem(*args)
    A = hn.Csr(args[0], args[1], rp, ci, val)
    assert_transpose_equal(A, O.transposed(rp, ci, val, args[1]))


def test_transpose_single_column_many_rows(hn):
    m = 300000  # one column spread over many radix tiles
    rp = np.arange(m + 1, dtype=np.int64)
    ci = np.zeros(m, dtype=np.int64)
    val = np.arange(1, m + 1, dtype=np.float64)
    A = hn.Csr(m, 1, rp, ci, val)
    assert_transpose_equal(A, O.transposed(rp, ci, val, 1))


def test_tile_tables_match_oracle(hn):
    lp = lpgen.lp_uniform(2000, 5000, 8, seed=0)
    A = hn.Csr(2000, 5000, lp["rp"], lp["ci"], lp["val"])
    for trans in (0, 1):
        items, row, nz = A.tiles(trans)
        rp = lp["rp"] if not trans else O.transposed(lp["rp"], lp["ci"], lp["val"], 5000)[0]
        rows = A.n if trans else A.m
        nnz = int(rp[-1])
        nt = (rows + nnz + items - 1) // items
        row_ref, nz_ref = O.merge_tiles(rp.astype(np.int32), nnz, items, nt)
        assert np.array_equal(row, row_ref) and np.array_equal(nz, nz_ref)


def test_set_values_rebuilds_transpose(hn):
    rp, ci, val, x = R.make_problem(300, 800, 0.08, 4242)
    A = hn.Csr(300, 800, rp, ci, val)
    val2 = val * -3.0
    val2[::5] = 0.0  # zeros now drop out of A^T
    A.set_values(val2)
    assert_transpose_equal(A, O.transposed(rp, ci, val2, 800))
    R.expect_close(A.spmv_host(x), O.multiply(rp, ci, val2, x), 1e-12)


def test_double_transpose_identity_large(hn):
    lp = lpgen.lp_zipf(seed=1000)
    A = hn.Csr(lp["m"], lp["n"], lp["rp"], lp["ci"], lp["val"])
    rpT, ciT, valT = A.export(trans=1)
    At = hn.Csr(lp["n"], lp["m"], rpT, ciT, valT)
    rp2, ci2, val2 = At.export(trans=1)
    assert np.array_equal(rp2.astype(np.int64), lp["rp"])
    assert np.array_equal(ci2.astype(np.int64), lp["ci"])
    assert np.array_equal(val2, lp["val"])
    # column lengths of the Zipf LP: the A^T rows carry the skew
    lens = np.diff(rpT.astype(np.int64))
    assert lens.max() > 100 and np.median(lens) <= 4
