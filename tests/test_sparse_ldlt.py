"""Host sparse LDL^T (hn_sparse_ldlt_solve, hn_amd_order) -- the seat of the
reference's SparseCholesky (core/numerical/factorization.hpp:162-208).

Solutions are checked by residual and against the reference's own
SparseCholesky (oracle/_ref) and a dense solve; the ordering is checked to be
a permutation whose fill is no worse than the reference's minimum degree on
structured and normal-equation matrices; the pivot clamp (d <= tol -> tol)
reports singular matrices as the reference does.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import lpgen
import oracle


@pytest.fixture(scope="module")
def hn():
    """The bindings without a device: the factorisation is host code."""
    import hnb200

    return hnb200


def csr(M):
    M = sp.csr_matrix(M)
    M.sum_duplicates()
    M.sort_indices()
    return M.indptr.astype(np.uint64), M.indices.astype(np.uint64), M.data.astype(np.float64)


def grid(k, shift=1e-3):
    T = sp.diags([-1.0, 2.0, -1.0], [-1, 0, 1], shape=(k, k))
    I = sp.eye(k)
    return (sp.kron(T, I) + sp.kron(I, T) + shift * sp.eye(k * k)).tocsr()


def normal_matrix(m, n, seed, spread=1.0):
    lp = lpgen.lp_uniform(m, n, 6, seed=seed)
    A = sp.csr_matrix((lp["val"], lp["ci"].astype(np.int64), lp["rp"].astype(np.int64)), shape=(m, n))
    rng = np.random.default_rng(seed)
    d = 10.0 ** rng.uniform(-spread, spread, n)  # IPM-like scaling spread
    return (A @ sp.diags(d) @ A.T + 1e-8 * sp.eye(m)).tocsr()


def staircase_normal(periods, k, seed):
    """Normal matrix of a multi-period LP: block tridiagonal."""
    rng = np.random.default_rng(seed)
    m, rows, cols, vals = periods * k, [], [], []
    j = 0
    for t in range(periods):
        for _ in range(2 * k):
            own = rng.choice(k, 4, replace=False) + t * k
            nxt = (rng.choice(k, 2, replace=False) + (t + 1) * k) if t + 1 < periods else []
            for r in list(own) + list(nxt):
                rows.append(r)
                cols.append(j)
                vals.append(rng.uniform(0.1, 1.0) * rng.choice([-1, 1]))
            j += 1
    A = sp.csr_matrix((vals, (rows, cols)), shape=(m, j))
    return (A @ sp.diags(rng.uniform(0.5, 2.0, j)) @ A.T + 1e-8 * sp.eye(m)).tocsr()


MATRICES = {
    "grid25": lambda: grid(25),
    "grid60": lambda: grid(60),
    "normal300": lambda: normal_matrix(300, 750, 3),
    "normal300_spread": lambda: normal_matrix(300, 750, 5, spread=6.0),
    "staircase": lambda: staircase_normal(40, 30, 7),
    "block_diag": lambda: sp.block_diag([grid(6), normal_matrix(40, 100, 2), sp.eye(17) * 3.0]).tocsr(),
}


@pytest.mark.parametrize("name", sorted(MATRICES))
def test_solution_residual_and_dense_agreement(hn, name):
    M = MATRICES[name]()
    rp, ci, v = csr(M)
    rng = np.random.default_rng(0)
    B = rng.standard_normal((3, M.shape[0]))
    X, st = hn.sparse_ldlt_solve(rp, ci, v, B)
    assert not st["singular"]
    for b, x in zip(B, X):
        assert np.linalg.norm(M @ x - b) <= 1e-11 * np.linalg.norm(b) * max(1.0, np.abs(M).max())
    if M.shape[0] <= 1000:
        Xd = np.linalg.solve(M.toarray(), B.T).T
        assert np.abs(X - Xd).max() <= 1e-8 * np.abs(Xd).max()


@pytest.mark.skipif(oracle.ref() is None, reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("name", ["grid25", "normal300", "staircase", "block_diag"])
def test_matches_reference_sparse_cholesky(hn, name):
    """Same solution as the reference's SparseCholesky (analyze, factorize,
    solve) and no more fill than its minimum-degree ordering (+5 %); the
    reference counts L's unit diagonal, this library does not."""
    M = MATRICES[name]()
    rp, ci, v = csr(M)
    b = np.sin(np.arange(M.shape[0]) + 1.0)
    ref = oracle.ref_cholesky_stats(rp, ci, v, b)
    x, st = hn.sparse_ldlt_solve(rp, ci, v, b)
    assert np.abs(x - ref["x"]).max() <= 1e-9 * np.abs(ref["x"]).max()
    assert st["nnz_L"] + M.shape[0] <= 1.05 * ref["nnz_L"]


def test_ordering_is_a_permutation_and_dense_rows_go_last(hn):
    n = 3000
    M = sp.lil_matrix((n, n))
    M.setdiag(4.0)
    M[0, 1:] = 1e-3  # a dense row and column
    M[1:, 0] = 1e-3
    for i in range(1, n - 1):
        M[i, i + 1] = M[i + 1, i] = -1.0
    rp, ci, v = csr(M)
    p = hn.amd_order(rp, ci)
    assert sorted(p.tolist()) == list(range(n))
    assert p[-1] == 0
    x, st = hn.sparse_ldlt_solve(rp, ci, v, np.ones(n))
    assert np.linalg.norm(M.tocsr() @ x - 1.0) <= 1e-12 * np.sqrt(n)
    assert st["nnz_L"] < 3 * n  # the chain and the dense row, no fill beyond


def test_singular_matrix_is_clamped_and_reported(hn):
    """A zero row and column (PSD, singular): the pivot is clamped to the
    tolerance and the factorisation reports it, as the reference does."""
    M = grid(12).tolil()
    M[30, :] = 0.0
    M[:, 30] = 0.0
    M = M.tocsr()
    rp, ci, v = csr(M)
    b = np.ones(M.shape[0])
    b[30] = 0.0
    x, st = hn.sparse_ldlt_solve(rp, ci, v, b, singular_tol=1e-12)
    assert st["singular"] and np.all(np.isfinite(x))
    mask = np.arange(M.shape[0]) != 30
    assert np.linalg.norm((M @ x - b)[mask]) <= 1e-10 * np.linalg.norm(b)
    if oracle.ref() is not None:
        assert oracle.ref_cholesky_stats(rp, ci, v)["singular"]


@pytest.mark.parametrize("m", [0, 1, 2])
def test_tiny_sizes(hn, m):
    M = sp.eye(m) * 2.0 if m else sp.csr_matrix((0, 0))
    rp, ci, v = csr(M)
    x, st = hn.sparse_ldlt_solve(rp, ci, v, np.ones(m))
    assert np.allclose(x, 0.5)


@pytest.mark.parametrize("name,build", [("normal3000", lambda: normal_matrix(3000, 7500, 11)),
                                        ("grid150", lambda: grid(150))])
def test_parallel_front_and_subtree_paths(hn, name, build):
    """Matrices large enough for the multithreaded paths: fronts wider than
    ~256 columns (the parallel trailing update of a front, here the
    3,000-row normal matrix of a random LP, which fills almost densely) and
    many independent subtrees (the 150 x 150 grid). Residuals as the smaller
    cases; the host library runs with the process's OpenMP threads (all cores
    unless OMP_NUM_THREADS says otherwise)."""
    M = build()
    rp, ci, v = csr(M)
    rng = np.random.default_rng(1)
    B = rng.standard_normal((2, M.shape[0]))
    X, st = hn.sparse_ldlt_solve(rp, ci, v, B)
    assert not st["singular"]
    for b, x in zip(B, X):
        assert np.linalg.norm(M @ x - b) <= 1e-10 * np.linalg.norm(b) * max(1.0, np.abs(M).max())
    if name == "grid150":
        assert st["supernodes"] > 1000
