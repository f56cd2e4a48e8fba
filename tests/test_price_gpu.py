"""GPU: revised-simplex pricing on the device against the oracle's
restatement of SimplexSolver's pricing (pinned to the reference in
test_price.py): reduced costs and Devex weights bit-identical, the entering
choice and the ranked shortlist identical (ties by lower index), dense columns
equal to extract_column."""
import numpy as np
import pytest

import lpgen
import oracle as O
from test_price import pricing_state

pytestmark = pytest.mark.gpu


def dev(torch, a, dtype=None):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda", dtype=dtype)


@pytest.mark.parametrize("shape", [(120, 300, 7), (2000, 5000, 21)])
def test_reduced_costs_bit_exact(hn, torch_cuda, shape):
    torch = torch_cuda
    m, n, seed = shape
    lp, y, cost, *_ = pricing_state(m, n, seed)
    A = hn.Csr(lp["m"], lp["n"], lp["rp"], lp["ci"], lp["val"])
    rc = torch.empty(n, dtype=torch.float64, device="cuda")
    hn.price_reduced_costs(A, dev(torch, y), dev(torch, cost), rc)
    torch.cuda.synchronize()
    want = O.price_reduced_costs(m, n, lp["rp"], lp["ci"], lp["val"], y, cost)
    assert np.array_equal(rc.cpu().numpy(), want)


@pytest.mark.parametrize("zero_u", [False, True])
def test_devex_update_bit_exact(hn, torch_cuda, zero_u):
    torch = torch_cuda
    lp, y, cost, nonbasis, artificial, w = pricing_state(400, 1000, 13)
    w = np.abs(np.nan_to_num(w, nan=1.0, posinf=1.0))
    u = np.zeros(lp["m"]) if zero_u else np.random.default_rng(4).standard_normal(lp["m"])
    u[::5] = 0.0
    A = hn.Csr(lp["m"], lp["n"], lp["rp"], lp["ci"], lp["val"])
    wd = dev(torch, w)
    alpha = torch.empty(lp["n"], dtype=torch.float64, device="cuda")
    hn.price_devex_update(A, dev(torch, u), dev(torch, nonbasis), wd, alpha)
    torch.cuda.synchronize()
    want_w, want_alpha = O.price_devex_update(lp["m"], lp["n"], lp["rp"], lp["ci"], lp["val"], u, nonbasis, w)
    assert np.array_equal(alpha.cpu().numpy(), want_alpha)
    assert np.array_equal(wd.cpu().numpy(), want_w)


@pytest.mark.parametrize("ties", [False, True])
@pytest.mark.parametrize("phase1,maximize", [(False, False), (True, False), (False, True)])
def test_select_matches_ranked_candidates(hn, torch_cuda, ties, phase1, maximize):
    torch = torch_cuda
    lp, y, cost, nonbasis, artificial, w = pricing_state(300, 800, 5, ties=ties)
    rc = O.price_reduced_costs(lp["m"], lp["n"], lp["rp"], lp["ci"], lp["val"], y, cost)
    if ties:
        rc = np.round(rc * 4) / 4
    n = lp["n"]
    args = (dev(torch, rc), dev(torch, w), dev(torch, nonbasis), dev(torch, artificial))
    k = 16
    out = torch.empty(k + 1, dtype=torch.int64, device="cuda")
    hn.price_select(n, *args, out, phase1=phase1, maximize=maximize, rule=hn.PRICE_RANKED, k=k)
    got = out.cpu().numpy()
    cnt, order = O.price_ranked(rc, w, nonbasis, artificial, phase1, maximize, cap=k)
    assert got[0] == cnt and cnt > k
    assert np.array_equal(got[1:], order)
    hn.price_select(n, *args, out, phase1=phase1, maximize=maximize, rule=hn.PRICE_BLAND)
    got = out.cpu().numpy()
    assert got[0] == cnt and got[1] == O.price_bland(rc, nonbasis, artificial, phase1, maximize)


def test_select_edge_cases(hn, torch_cuda):
    torch = torch_cuda
    n = 1000
    rng = np.random.default_rng(2)
    rc = np.abs(rng.standard_normal(n))  # nothing improving
    nb = np.arange(n, dtype=np.int32)
    out = torch.empty(5, dtype=torch.int64, device="cuda")
    hn.price_select(n, dev(torch, rc), None, dev(torch, nb), None, out, rule=hn.PRICE_RANKED, k=4)
    assert out.cpu().tolist() == [0, -1, -1, -1, -1]
    hn.price_select(n, dev(torch, rc), None, dev(torch, nb), None, out, rule=hn.PRICE_BLAND)
    assert out.cpu().tolist()[:2] == [0, -1]
    rc[[3, 700]] = -1.0  # two improving columns with equal score: index order
    hn.price_select(n, dev(torch, rc), None, dev(torch, nb), None, out, rule=hn.PRICE_RANKED, k=4)
    assert out.cpu().tolist() == [2, 3, 700, -1, -1]
    with pytest.raises(hn.HnError):
        hn.price_select(n, dev(torch, rc), None, dev(torch, nb), None, out, rule=hn.PRICE_RANKED, k=0)
    # empty problem
    hn.price_select(0, None, None, None, None, out, rule=hn.PRICE_RANKED, k=1)
    assert out.cpu().tolist()[:2] == [0, -1]


def test_columns_match_extract_column(hn, torch_cuda):
    torch = torch_cuda
    lp = lpgen.lp_uniform(500, 1250, 6, 8)
    A = hn.Csr(lp["m"], lp["n"], lp["rp"], lp["ci"], lp["val"])
    cols = np.array([0, 5, 1249, 600, 5], dtype=np.int64)
    out = torch.full((cols.size, lp["m"]), np.nan, dtype=torch.float64, device="cuda")
    hn.price_columns(A, dev(torch, cols), out)
    got = out.cpu().numpy()
    for r, j in enumerate(cols):
        assert np.array_equal(got[r], O.extract_column(lp["m"], lp["rp"], lp["ci"], lp["val"], int(j)))
    bad = dev(torch, np.array([1, 1250], dtype=np.int64))
    with pytest.raises(hn.HnError):
        hn.price_columns(A, bad, out[:2])
