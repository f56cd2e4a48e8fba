"""GPU parity: SpMV / A^T SpMV / SpMM through the C ABI against the oracle.

Inputs are the reference tests' own matrices (tests/unit/test_gpu_backend.cpp,
rebuilt bit-for-bit by refcases.py) with the reference's tolerances, the
synthetic LPs of the measured workloads, and the edge cases the reference
covers (empty matrix, empty rows) plus row lengths around warp/tile edges.
Tolerance: |y_i - y_ref_i| <= 1e-12 * sum_k |a_ik x_k| (normwise 1e-12).
"""
import numpy as np
import pytest

import lpgen
import oracle as O
import refcases as R

pytestmark = pytest.mark.gpu


def dev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def run_spmv(hn, torch, A, x, trans=0, alpha=1.0, beta=0.0, y0=None):
    rows = A.n if trans else A.m
    xd = dev(torch, x)
    yd = dev(torch, y0) if y0 is not None else torch.full((rows,), float("nan"), dtype=torch.float64, device="cuda")
    A.spmv(xd, yd, trans=trans, alpha=alpha, beta=beta)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


@pytest.mark.parametrize("args,tol", [((200, 150, 0.10, 42), 1e-12),     # :90-98
                                      ((1500, 1200, 0.003, 77), 1e-10),  # :211-222 scalar-kernel case
                                      ((300, 800, 0.08, 4242), 1e-10)])  # :224-234 warp-kernel case
def test_reference_spmv_cases(hn, torch_cuda, args, tol):
    rp, ci, val, x = R.make_problem(*args)
    A = hn.Csr(args[0], args[1], rp, ci, val)
    y_ref = O.multiply(rp, ci, val, x)
    y = run_spmv(hn, torch_cuda, A, x)
    R.expect_close(y, y_ref, tol)
    R.normwise_close(y, y_ref, rp, ci, val, x, 1e-12)
    R.expect_close(A.spmv_host(x), y_ref, tol)


def test_empty_rows(hn, torch_cuda):
    # CudaBackendTest.SpmvEmptyRows (:236-258): every 4th row of a 2*I empty
    n = 256
    keep = np.array([i % 4 != 0 for i in range(n)])
    rp = np.concatenate([[0], np.cumsum(keep)]).astype(np.int64)
    ci = np.flatnonzero(keep)
    A = hn.Csr(n, n, rp, ci, np.full(ci.shape[0], 2.0))
    y = run_spmv(hn, torch_cuda, A, np.full(n, 1.5))
    expected = np.where(keep, 3.0, 0.0)
    assert np.array_equal(y, expected)


def test_empty_matrix(hn, torch_cuda):
    # CpuBackendTest.EmptyMatrixIsSafe (:126-131)
    A = hn.Csr(0, 0, np.array([0]), np.zeros(0), np.zeros(0))
    assert A.spmv_host(np.zeros(0)).shape == (0,)
    B = hn.Csr(5, 3, np.zeros(6), np.zeros(0), np.zeros(0))
    assert np.array_equal(B.spmv_host(np.ones(3)), np.zeros(5))
    assert np.array_equal(B.spmv_host(np.ones(5), trans=1), np.zeros(3))


@pytest.mark.parametrize("lens", [[1], [31, 32, 33], [1024, 2000, 2047, 2048, 2049], [5000, 1, 0, 7],
                                  [0] * 3000 + [70000] + [3] * 5000])
def test_row_length_edges(hn, torch_cuda, lens):
    rng = np.random.default_rng(len(lens))
    n = 80000
    lens = np.array(lens, dtype=np.int64)
    rp = np.concatenate([[0], np.cumsum(lens)])
    ci = np.concatenate([np.sort(rng.choice(n, size=L, replace=False)) for L in lens]) if lens.sum() else np.zeros(0)
    val = rng.uniform(-1, 1, size=int(lens.sum()))
    x = rng.standard_normal(n)
    A = hn.Csr(len(lens), n, rp, ci, val)
    y = run_spmv(hn, torch_cuda, A, x)
    R.normwise_close(y, O.multiply(rp, ci, val, x), rp, ci, val, x)
    xt = rng.standard_normal(len(lens))
    yt = run_spmv(hn, torch_cuda, A, xt, trans=1)
    R.expect_close(yt, O.tmultiply(rp, ci, val, xt, n), 1e-12)


def test_alpha_beta(hn, torch_cuda):
    rp, ci, val, x = R.make_problem(300, 800, 0.08, 4242)
    A = hn.Csr(300, 800, rp, ci, val)
    y0 = np.random.default_rng(3).standard_normal(300)
    y = run_spmv(hn, torch_cuda, A, x, alpha=2.0, beta=-0.5, y0=y0)
    R.expect_close(y, 2.0 * O.multiply(rp, ci, val, x) - 0.5 * y0, 1e-12)


def test_transpose_product_reference_case(hn, torch_cuda):
    rp, ci, val, _ = R.make_problem(300, 800, 0.08, 4242)
    A = hn.Csr(300, 800, rp, ci, val)
    xt = R.uniform(11, 300, -4.0, 4.0)
    yt = run_spmv(hn, torch_cuda, A, xt, trans=1)
    # the reference's own output (golden) for this input
    gold = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden",
                                              "reference_golden.npz"))["tmul_300x800_y"]
    R.expect_close(yt, gold, 1e-12)


@pytest.mark.parametrize("args,k,bseed,lo,hi,tol", [((80, 60, 0.2, 7), 4, 99, -2.0, 2.0, 1e-10),        # :100-124
                                                    ((400, 300, 0.05, 2024), 5, 8, -1.0, 1.0, 1e-10),   # :260-277
                                                    ((4000, 3000, 0.08, 31337), 64, None, 1.0, 1.0, 1e-9)])  # :294-314
def test_reference_spmm_cases(hn, torch_cuda, args, k, bseed, lo, hi, tol):
    rp, ci, val, _ = R.make_problem(*args)
    B = R.uniform(bseed, args[1] * k, lo, hi) if bseed is not None else np.ones(args[1] * k)
    A = hn.Csr(args[0], args[1], rp, ci, val)
    C_ref = O.spmm(rp, ci, val, B, k)
    R.expect_close(A.spmm_host(B, k), C_ref, tol)
    Bd = dev(torch_cuda, B)
    Cd = torch_cuda.empty(args[0] * k, dtype=torch_cuda.float64, device="cuda")
    A.spmm(Bd, k, Cd)
    torch_cuda.cuda.synchronize()
    R.expect_close(Cd.cpu().numpy(), C_ref, tol)


def test_spmm_transposed(hn, torch_cuda):
    rp, ci, val, _ = R.make_problem(400, 300, 0.05, 2024)
    A = hn.Csr(400, 300, rp, ci, val)
    k = 130
    B = np.random.default_rng(1).standard_normal(400 * k)
    rpT, ciT, valT = O.transposed(rp, ci, val, 300)
    R.expect_close(A.spmm_host(B, k, trans=1), O.spmm(rpT, ciT, valT, B, k), 1e-12)


def test_deterministic_bits(hn, torch_cuda):
    lp = lpgen.lp_uniform(2000, 5000, 8, seed=0)
    A = hn.Csr(2000, 5000, lp["rp"], lp["ci"], lp["val"])
    x = np.random.default_rng(0).standard_normal(5000)
    ys = [run_spmv(hn, torch_cuda, A, x) for _ in range(3)]
    assert all(np.array_equal(ys[0], y) for y in ys[1:])


def test_lp_config0_shape(hn, torch_cuda):
    lp = lpgen.lp_uniform(2000, 5000, 8, seed=0)
    rp, ci, val = lp["rp"], lp["ci"], lp["val"]
    A = hn.Csr(2000, 5000, rp, ci, val)
    y = run_spmv(hn, torch_cuda, A, lp["x0"])
    R.normwise_close(y, O.multiply(rp, ci, val, lp["x0"]), rp, ci, val, lp["x0"])
    yt = run_spmv(hn, torch_cuda, A, lp["y0"], trans=1)
    yt_ref = O.matvec_t(rp, ci, val, lp["y0"], 5000)
    rpT, ciT, valT = O.transposed(rp, ci, val, 5000)
    R.normwise_close(yt, yt_ref, rpT, ciT, valT, lp["y0"])


@pytest.fixture(scope="module")
def big_lp():
    """The m=200k, n=500k Zipf(1.5) LP at ~5.2M nonzeros."""
    return lpgen.lp_zipf(seed=1000)


def test_large_zipf_lp_parity(hn, torch_cuda, big_lp):
    lp = big_lp
    rp, ci, val = lp["rp"], lp["ci"], lp["val"]
    A = hn.Csr(lp["m"], lp["n"], rp, ci, val)
    assert A.nnz > 4_500_000
    y = run_spmv(hn, torch_cuda, A, lp["x0"])
    R.normwise_close(y, O.multiply(rp, ci, val, lp["x0"]), rp, ci, val, lp["x0"])
    yt = run_spmv(hn, torch_cuda, A, lp["y0"], trans=1)
    rpT, ciT, valT = O.transposed(rp, ci, val, lp["n"])
    R.normwise_close(yt, O.matvec_t(rp, ci, val, lp["y0"], lp["n"]), rpT, ciT, valT, lp["y0"])
    # size-independent property: 1^T (A x) == (A^T 1)^T x to rounding
    ones = np.ones(lp["m"])
    at1 = run_spmv(hn, torch_cuda, A, ones, trans=1)
    lhs, rhs = y.sum(), at1 @ lp["x0"]
    assert abs(lhs - rhs) <= 1e-10 * (np.abs(val).sum() * 2.0)


@pytest.mark.parametrize("kind,t", [(None, None), (0, 0), (1, 4), (1, 16)])
def test_spec_literal_zipf_lp_parity(hn, torch_cuda, kind, t):
    """The spec-literal large LP: m 200k, n 500k, Zipf(1.5) column counts on
    [1, 2000] without rescaling (about 17M nonzeros). y = A x and A^T y on the
    autotuned path and on each path pinned, normwise 1e-12 against the
    oracle's multiply / matvec_t."""
    lp = lpgen.lp_zipf(seed=1000, target_nnz=None)
    rp, ci, val = lp["rp"], lp["ci"], lp["val"]
    A = hn.Csr(lp["m"], lp["n"], rp, ci, val)
    assert A.nnz > 15_000_000
    if kind is not None:
        A.set_spmv_kind(kind, t, trans=0)
        A.set_spmv_kind(kind, t, trans=1)
    y = run_spmv(hn, torch_cuda, A, lp["x0"])
    R.normwise_close(y, O.multiply(rp, ci, val, lp["x0"]), rp, ci, val, lp["x0"])
    yt = run_spmv(hn, torch_cuda, A, lp["y0"], trans=1)
    rpT, ciT, valT = O.transposed(rp, ci, val, lp["n"])
    R.normwise_close(yt, O.matvec_t(rp, ci, val, lp["y0"], lp["n"]), rpT, ciT, valT, lp["y0"])
