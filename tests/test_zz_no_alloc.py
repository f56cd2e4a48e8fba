"""GPU: hn_spmv_noalloc, the SpMV entry point that allocates no device memory.

It serves callers that cannot call cudaMalloc -- a solver living inside a
framework whose memory pool owns the device, or an IPM / branch-and-bound loop
that must not allocate mid-solve. Its scratch is a fixed __device__ array, so
this test checks, through the C ABI, that two calls in a row agree with the
allocating entry point hn_spmv (normwise 1e-12, the SpMV tolerance of these
tests) and that sizes beyond the array are refused. This file is collected
last so a failure here stops a -x run only after every other test ran.
"""
import numpy as np
import pytest

import lpgen
import refcases as R

pytestmark = pytest.mark.gpu


def device_csr(torch, rp, ci, val):
    return (torch.as_tensor(np.asarray(rp, dtype=np.int32), device="cuda"),
            torch.as_tensor(np.asarray(ci, dtype=np.int32), device="cuda"),
            torch.as_tensor(np.asarray(val, dtype=np.float64), device="cuda"))


def noalloc(hn, torch, m, n, rp_d, ci_d, val_d, x):
    y = torch.full((m,), float("nan"), dtype=torch.float64, device="cuda")
    hn.check(hn.load().hn_spmv_noalloc(m, n, ci_d.numel(), rp_d.data_ptr(), ci_d.data_ptr(), val_d.data_ptr(),
                                       x.data_ptr(), y.data_ptr(), None))
    torch.cuda.synchronize()
    return y.cpu().numpy()


@pytest.mark.parametrize("case", ["reference_300x800", "lp_2000x5000", "zipf_200k"])
def test_noalloc_matches_allocating_spmv_twice(hn, torch_cuda, case):
    torch = torch_cuda
    if case == "reference_300x800":
        rp, ci, val, x = R.make_problem(300, 800, 0.08, 4242)
        m, n = 300, 800
        x2 = x[::-1].copy()
    else:
        lp = lpgen.lp_uniform(2000, 5000, 8, 0) if case == "lp_2000x5000" else lpgen.lp_zipf(seed=1000)
        rp, ci, val, m, n = lp["rp"], lp["ci"], lp["val"], lp["m"], lp["n"]
        x, x2 = lp["x0"], np.random.default_rng(1).standard_normal(n)
    A = hn.Csr(m, n, rp, ci, val)
    rp_d, ci_d, val_d = device_csr(torch, rp, ci, val)
    for xv in (x, x2):  # two calls in a row: the shared scratch keeps the last call's contents
        xd = torch.as_tensor(xv, device="cuda")
        y_ref = torch.empty(m, dtype=torch.float64, device="cuda")
        A.spmv(xd, y_ref)
        y = noalloc(hn, torch, m, n, rp_d, ci_d, val_d, xd)
        R.normwise_close(y, y_ref.cpu().numpy(), rp, ci, val, xv, 1e-12)


def test_noalloc_refuses_sizes_beyond_scratch(hn, torch_cuda):
    torch = torch_cuda
    rp_d = torch.zeros(2, dtype=torch.int32, device="cuda")
    with pytest.raises(hn.HnError) as e:
        hn.check(hn.load().hn_spmv_noalloc(1, 1, 117440512, rp_d.data_ptr(), rp_d.data_ptr(), rp_d.data_ptr(),
                                           rp_d.data_ptr(), rp_d.data_ptr(), None))
    assert e.value.status == hn.HN_ERR_INVALID_ARG and "scratch limit" in str(e.value)
