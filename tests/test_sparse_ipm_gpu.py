"""The GPU IPM with the host sparse LDL^T (SparseLDLT) as its normal-matrix
factorisation.

(a) Forced sparse against the dense LDL^T on the same LP: same status,
objective within the IPM tolerance. (b) A staircase LP above the dense
limit (12,600 rows, automatic choice = sparse): OPTIMAL, with its KKT
residuals checked on the original LP through the returned primal x and the
barrier's dual estimate (y, s).
"""
import numpy as np
import pytest
import scipy.sparse as sp

import lpgen

pytestmark = pytest.mark.gpu


def test_sparse_and_dense_factorisations_agree(hn):
    lp = lpgen.lp_uniform(300, 750, 6, seed=11)
    dense = hn.lp_solve(lp, factorization=1)
    sparse = hn.lp_solve(lp, factorization=2)
    assert dense["status_name"] == sparse["status_name"] == "OPTIMAL"
    assert abs(sparse["objective"] - dense["objective"]) <= 1e-8 * (1.0 + abs(dense["objective"]))
    assert abs(sparse["iterations"] - dense["iterations"]) <= 2


def test_staircase_lp_above_the_dense_limit_is_solved(hn):
    lp = lpgen.lp_staircase(210, 60, seed=1)
    r = hn.lp_solve(lp)  # 12,600 rows: the automatic choice is the sparse factorisation
    assert r["status_name"] == "OPTIMAL", r["error"]
    A = sp.csr_matrix((lp["val"], lp["ci"].astype(np.int64), lp["rp"].astype(np.int64)), shape=(lp["m"], lp["n"]))
    x, y, s, b, c = r["x"], r["y"], r["s"], lp["b"], lp["c"]
    assert np.all(x >= -1e-9)
    assert np.abs(A @ x - b).max() <= 1e-6 * (1.0 + np.abs(b).max())
    assert np.abs(A.T @ y + s - c).max() <= 1e-6 * (1.0 + np.abs(c).max())
    assert abs(c @ x - b @ y) <= 1e-6 * (1.0 + abs(c @ x))
