"""GPU: the two SpMV paths (merge-path tiles and the row-length-binned
vector kernel) on A and on the device A^T, against the oracle's
SparseMatrix::multiply / transpose_multiply restatement (normwise 1e-12),
the IPM's residual epilogues through hn_ipm_residuals; the autotuner's
choice; bins rebuilt after hn_csr_set_values."""
import numpy as np
import pytest

import lpgen
import oracle as O
import refcases as R

pytestmark = pytest.mark.gpu

PATHS = [(0, 0), (1, 1), (1, 4), (1, 16)]


def dev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def normwise_ok(y, y_ref, rp, ci, val, x, tol=1e-12):
    absr = O.multiply(rp, ci, np.abs(val), np.abs(x))
    return np.all(np.abs(y - y_ref) <= tol * absr + 1e-300)


def ragged_matrix(seed=3):
    """Rows of length 0, 1, 2..40, a few of 300 and 1500 (past 32 lanes x t)."""
    rng = np.random.default_rng(seed)
    n = 2000
    lens = np.concatenate([np.zeros(40, int), rng.integers(1, 41, 500), [300, 1500, 0, 1, 1500, 33, 64, 65]])
    rng.shuffle(lens)
    rows = [np.sort(rng.choice(n, size=L, replace=False)) for L in lens]
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    ci = np.concatenate(rows).astype(np.int64)
    val = rng.uniform(-1, 1, ci.size)
    return len(lens), n, rp, ci, val


@pytest.mark.parametrize("kind,t", PATHS)
def test_paths_match_oracle_on_ragged_rows(hn, torch_cuda, kind, t):
    m, n, rp, ci, val = ragged_matrix()
    A = hn.Csr(m, n, rp, ci, val, autotune=False)
    A.set_spmv_kind(kind, t, trans=0)
    A.set_spmv_kind(kind, t, trans=1)
    assert A.spmv_kind(0) == (kind, t if kind else 0) and A.spmv_kind(1) == (kind, t if kind else 0)
    rng = np.random.default_rng(1)
    x, lam = rng.standard_normal(n), rng.standard_normal(m)
    y = torch_cuda.full((m,), float("nan"), dtype=torch_cuda.float64, device="cuda")
    A.spmv(dev(torch_cuda, x), y)
    assert normwise_ok(y.cpu().numpy(), O.multiply(rp, ci, val, x), rp, ci, val, x)
    t_ = torch_cuda.full((n,), float("nan"), dtype=torch_cuda.float64, device="cuda")
    A.spmv(dev(torch_cuda, lam), t_, trans=1)
    rpT, ciT, valT = O.transposed(rp, ci, val, n)
    assert normwise_ok(t_.cpu().numpy(), O.tmultiply(rp, ci, val, lam, n), rpT, ciT, valT, lam)
    # residual y = A x - b
    bb = rng.standard_normal(m)
    yr = torch_cuda.full((m,), float("nan"), dtype=torch_cuda.float64, device="cuda")
    A.residual(dev(torch_cuda, x), dev(torch_cuda, bb), yr)
    ref = O.multiply(rp, ci, val, x) - bb
    assert np.all(np.abs(yr.cpu().numpy() - ref) <= 1e-12 * O.multiply(rp, ci, np.abs(val), np.abs(x)) + 1e-16 * np.abs(bb))
    # alpha/beta epilogue
    y0 = rng.standard_normal(m)
    yd = dev(torch_cuda, y0)
    A.spmv(dev(torch_cuda, x), yd, alpha=-2.0, beta=0.5)
    ref = -2.0 * O.multiply(rp, ci, val, x) + 0.5 * y0
    assert np.all(np.abs(yd.cpu().numpy() - ref) <= 2e-12 * (O.multiply(rp, ci, np.abs(val), np.abs(x)) + np.abs(y0)))


def test_ipm_residual_epilogues_on_binned_path(hn, torch_cuda):
    """hn_ipm_residuals (y = Mx - b, rd = M^T lam + z - c) on the binned path
    against the oracle."""
    lp = lpgen.lp_uniform(300, 750, 8, 9)
    m, n = lp["m"], lp["n"]
    A = hn.Csr(m, n, lp["rp"], lp["ci"], lp["val"], autotune=False)
    A.set_spmv_kind(1, 4, trans=0)
    A.set_spmv_kind(1, 8, trans=1)
    rng = np.random.default_rng(2)
    x, z, lam = rng.uniform(0.5, 2, n), rng.uniform(0.5, 2, n), rng.standard_normal(m)
    T = torch_cuda
    d = {k: dev(T, v) for k, v in dict(x=x, z=z, lam=lam, b=lp["b"], c=lp["c"]).items()}
    out = {k: T.empty(sz, dtype=T.float64, device="cuda") for k, sz in
           dict(mx=m, rp=m, rd=n, D=n, Drd=n).items()}
    scal = T.zeros(8, dtype=T.float64, device="cuda")
    hn.check(hn.load().hn_ipm_residuals(A.h, d["x"].data_ptr(), d["lam"].data_ptr(), d["z"].data_ptr(),
                                        d["b"].data_ptr(), d["c"].data_ptr(), out["mx"].data_ptr(),
                                        out["rp"].data_ptr(), out["rd"].data_ptr(), out["D"].data_ptr(),
                                        out["Drd"].data_ptr(), scal.data_ptr(), None))
    T.cuda.synchronize()
    mx = O.multiply(lp["rp"], lp["ci"], lp["val"], x)
    absr = O.multiply(lp["rp"], lp["ci"], np.abs(lp["val"]), np.abs(x))
    assert np.all(np.abs(out["mx"].cpu().numpy() - mx) <= 1e-12 * absr)
    assert np.all(np.abs(out["rp"].cpu().numpy() - (mx - lp["b"])) <= 1e-12 * absr + 1e-15 * np.abs(lp["b"]))
    mtl = O.matvec_t(lp["rp"], lp["ci"], lp["val"], lam, n)
    absd = O.matvec_t(lp["rp"], lp["ci"], np.abs(lp["val"]), np.abs(lam), n)
    assert np.all(np.abs(out["rd"].cpu().numpy() - ((mtl + z) - lp["c"])) <= 1e-12 * (absd + np.abs(z) + np.abs(lp["c"])))


@pytest.fixture(scope="module")
def big_lp():
    """The m=200k, n=500k Zipf(1.5) LP at ~5.2M nonzeros (autotuned size)."""
    return lpgen.lp_zipf(seed=1000)


def test_autotune_choice_and_set_values(hn, torch_cuda, big_lp):
    lp = big_lp
    m, n = lp["m"], lp["n"]
    A = hn.Csr(m, n, lp["rp"], lp["ci"], lp["val"])
    for d in (0, 1):
        k, t = A.spmv_kind(d)
        assert (k, t) in {(0, 0), (1, 4), (1, 8), (1, 16)}
    # A^T bins follow a value update that drops exact zeros
    val = np.array(lp["val"], dtype=np.float64)
    val[::97] = 0.0
    A.set_spmv_kind(1, 8, trans=1)
    A.set_values(val)
    assert A.spmv_kind(1) == (1, 8)
    rng = np.random.default_rng(3)
    lam = rng.standard_normal(m)
    t_ = torch_cuda.empty(n, dtype=torch_cuda.float64, device="cuda")
    A.spmv(dev(torch_cuda, lam), t_, trans=1)
    rpT, ciT, valT = O.transposed(lp["rp"], lp["ci"], val, n)
    assert normwise_ok(t_.cpu().numpy(), O.tmultiply(lp["rp"], lp["ci"], val, lam, n), rpT, ciT, valT, lam)
