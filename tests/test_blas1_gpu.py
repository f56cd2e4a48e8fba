"""GPU: dot / axpy / norms (IComputeBackend::dot/axpy/norm_inf,
core/execution/gpu_backend.cpp:123-134) against the oracle, plus the error
behaviour of the C ABI (status codes, no CPU fallback, host fault injection)."""
import ctypes as C

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [0, 1, 1000, 12345, 3_000_001])
def test_dot_nrm_axpy(hn, torch_cuda, n):
    torch = torch_cuda
    rng = np.random.default_rng(n)
    a, b = rng.standard_normal(n), rng.standard_normal(n)
    ad, bd = torch.as_tensor(a, device="cuda"), torch.as_tensor(b, device="cuda")
    out = torch.empty(4, dtype=torch.float64, device="cuda")
    hn.dot(n, ad, bd, out[0:1])
    hn.nrm2(n, ad, out[1:2])
    hn.nrm_inf(n, ad, out[2:3])
    hn.axpy(n, 0.75, ad, bd)
    torch.cuda.synchronize()
    r = out.cpu().numpy()
    assert abs(r[0] - O.dot(a, b)) <= 1e-12 * np.abs(a * b).sum()
    assert abs(r[1] - O.nrm2(a)) <= 1e-12 * max(O.nrm2(a), 1e-300)
    assert r[2] == O.norm_inf(a)
    assert np.array_equal(bd.cpu().numpy(), O.axpy(0.75, a, b))


def test_norm_inf_ignores_nan_like_reference(hn, torch_cuda):
    torch = torch_cuda
    v = np.array([1.0, np.nan, -7.5, 3.0])
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    hn.nrm_inf(4, torch.as_tensor(v, device="cuda"), out)
    assert out.item() == O.norm_inf(v) == 7.5


def test_reductions_deterministic(hn, torch_cuda):
    torch = torch_cuda
    a = torch.randn(5_000_000, dtype=torch.float64, device="cuda")
    out = torch.empty(3, dtype=torch.float64, device="cuda")
    for i in range(3):
        hn.dot(a.numel(), a, a, out[i:i + 1])
    torch.cuda.synchronize()
    assert out[0].item() == out[1].item() == out[2].item()


def test_invalid_csr_rejected_before_gpu(hn):
    with pytest.raises(hn.HnError) as e:
        hn.Csr(2, 3, np.array([0, 1, 2]), np.array([0, 3]), np.array([1.0, 1.0]))
    assert e.value.status == hn.HN_ERR_INVALID_ARG and "out of range" in str(e.value)
    with pytest.raises(hn.HnError):
        hn.Csr(2, 3, np.array([0, 2, 1]), np.array([0, 1]), np.array([1.0, 1.0]))
    with pytest.raises(hn.HnError):
        hn.Csr(2, 3, np.array([1, 2, 2]), np.array([0, 1]), np.array([1.0, 1.0]))


def test_fault_injection_then_recovery(hn, torch_cuda):
    A = hn.Csr(3, 3, np.array([0, 1, 2, 3]), np.array([0, 1, 2]), np.array([1.0, 2.0, 3.0]))
    hn.fault_inject(0, hn.HN_ERR_INJECTED)
    with pytest.raises(hn.HnError) as e:
        A.spmv_host(np.ones(3))
    assert e.value.status == hn.HN_ERR_INJECTED
    assert np.array_equal(A.spmv_host(np.ones(3)), np.array([1.0, 2.0, 3.0]))


def test_missing_transpose_is_an_error(hn):
    A = hn.Csr(3, 3, np.array([0, 1, 2, 3]), np.array([0, 1, 2]), np.ones(3), transpose=False)
    with pytest.raises(hn.HnError):
        A.spmv_host(np.ones(3), trans=1)


def test_kernel_counter_advances(hn, torch_cuda):
    A = hn.Csr(3, 3, np.array([0, 1, 2, 3]), np.array([0, 1, 2]), np.ones(3))
    before, _ = hn.stats()
    A.spmv_host(np.ones(3))
    after, _ = hn.stats()
    assert after > before


def test_device_info(hn):
    d = hn.device_info()
    assert d.cc_major == 10 and d.sm_count > 0 and d.total_mem > 0
