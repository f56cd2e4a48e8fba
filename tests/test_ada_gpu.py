"""GPU: A diag(d) A^T assembly against build_normal_equations
(core/lp/interior_point.cpp:144-200) restated by the oracle and, for one
case, assembled by the reference's own from_triplets (golden fixture).

Pattern: bit-exact. Values: |N_ik - ref_ik| <= 1e-12 * (|A| D |A|^T)_ik + the
regularisation term (the reference sums duplicate triplets in an order its
std::sort leaves open). dyn_reg: exactly equal (the diagonal is summed in
the same column order on both sides).
"""
import os

import numpy as np
import pytest

import lpgen
import oracle as O

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_golden.npz"))


def assemble(hn, torch, lp, D, reg=1e-8, compact=False):
    A = hn.Csr(lp["m"], lp["n"], lp["rp"], lp["ci"], lp["val"])
    P = hn.Pattern(A, compact=compact)
    nval = torch.empty(P.nnz, dtype=torch.float64, device="cuda")
    dyn = torch.empty(1, dtype=torch.float64, device="cuda")
    Dd = torch.as_tensor(D, device="cuda")
    P.numeric(Dd, reg, nval, dyn)
    torch.cuda.synchronize()
    rp, ci = P.export()
    return A, P, rp.astype(np.int64), ci.astype(np.int64), nval.cpu().numpy(), float(dyn.item())


def check_values(lp, D, reg, rp, ci, vals, dyn):
    rpR, ciR, vR, dynR = O.normal_equations(lp["rp"], lp["ci"], lp["val"], D, reg, lp["n"])
    _, _, absR, _ = O.normal_equations(lp["rp"], lp["ci"], np.abs(lp["val"]), D, 0.0, lp["n"])
    assert dyn == dynR
    # map reference entries into the device pattern (device pattern is a superset)
    m = lp["m"]
    key = np.repeat(np.arange(m), np.diff(rp)) * m + ci
    keyR = np.repeat(np.arange(m), np.diff(rpR)) * m + ciR
    pos = np.searchsorted(key, keyR)
    assert np.array_equal(key[pos], keyR)
    assert np.all(np.abs(vals[pos] - vR) <= 1e-12 * (absR + dynR))
    extra = np.ones(key.shape[0], dtype=bool)
    extra[pos] = False
    assert np.all(vals[extra] == 0.0)  # entries only inactive columns reach stay explicit zeros


@pytest.mark.parametrize("m,n,k,seed", [(200, 500, 8, 11), (2000, 5000, 8, 0), (529, 1322, 6, 7)])
def test_pattern_and_values_all_active(hn, torch_cuda, m, n, k, seed):
    lp = lpgen.scaled_problem(lpgen.lp_uniform(m, n, k, seed))
    D = np.random.default_rng(seed).uniform(1e-3, 1e3, n)
    A, P, rp, ci, vals, dyn = assemble(hn, torch_cuda, lp, D)
    rpP, ciP = O.ada_pattern(lp["rp"], lp["ci"], n)
    assert np.array_equal(rp, rpP) and np.array_equal(ci, ciP.astype(np.int64))
    check_values(lp, D, 1e-8, rp, ci, vals, dyn)


def test_inactive_columns_and_reference_golden(hn, torch_cuda):
    lp = lpgen.scaled_problem(lpgen.lp_uniform(200, 500, 8, seed=11))
    D = GOLD["ne_D"]  # every 9th column inactive (D_j = 0)
    A, P, rp, ci, vals, dyn = assemble(hn, torch_cuda, lp, D)
    assert dyn == GOLD["ne_dyn"][0]
    check_values(lp, D, 1e-8, rp, ci, vals, dyn)
    # against the reference's own assembly (from_triplets of its triplets)
    m = 200
    key = np.repeat(np.arange(m), np.diff(rp)) * m + ci
    rpG, ciG, vG = GOLD["ne_rp"].astype(np.int64), GOLD["ne_ci"].astype(np.int64), GOLD["ne_val"]
    keyG = np.repeat(np.arange(m), np.diff(rpG)) * m + ciG
    pos = np.searchsorted(key, keyG)
    assert np.array_equal(key[pos], keyG)
    _, _, absR, _ = O.normal_equations(lp["rp"], lp["ci"], np.abs(lp["val"]), D, 0.0, 500)
    assert np.all(np.abs(vals[pos] - vG) <= 1e-12 * (absR + dyn))


def test_dynamic_regularisation_dominates(hn, torch_cuda):
    lp = lpgen.scaled_problem(lpgen.lp_uniform(200, 500, 8, seed=3))
    D = np.full(500, 1e9)  # 1e-12 * max diag >> reg
    *_, rp, ci, vals, dyn = assemble(hn, torch_cuda, lp, D, reg=1e-8)
    assert dyn > 1e-8
    check_values(lp, D, 1e-8, rp, ci, vals, dyn)


def test_repeat_numeric_is_deterministic(hn, torch_cuda):
    lp = lpgen.scaled_problem(lpgen.lp_uniform(2000, 5000, 8, 0))
    D = np.random.default_rng(1).uniform(0.1, 10, 5000)
    A = hn.Csr(2000, 5000, lp["rp"], lp["ci"], lp["val"])
    P = hn.Pattern(A)
    Dd = torch_cuda.as_tensor(D, device="cuda")
    outs = []
    for _ in range(3):
        nval = torch_cuda.empty(P.nnz, dtype=torch_cuda.float64, device="cuda")
        P.numeric(Dd, 1e-8, nval)
        outs.append(nval.cpu().numpy())
    assert all(np.array_equal(outs[0], o) for o in outs[1:])


def test_large_zipf_pattern_properties(hn, torch_cuda):
    """Full 200k x 500k size: pattern symmetric with a full diagonal, and
    N x == A (D (A^T x)) to rounding for random x (a size-independent check)."""
    lp = lpgen.scaled_problem(lpgen.lp_zipf(seed=1000))
    m, n = lp["m"], lp["n"]
    torch = torch_cuda
    A = hn.Csr(m, n, lp["rp"], lp["ci"], lp["val"])
    P = hn.Pattern(A)
    D = torch.rand(n, dtype=torch.float64, device="cuda") + 0.5
    nval = torch.empty(P.nnz, dtype=torch.float64, device="cuda")
    dyn = torch.empty(1, dtype=torch.float64, device="cuda")
    P.numeric(D, 1e-8, nval, dyn)
    rp_d, ci_d, dp_d = P.device_arrays()
    rp, ci = P.export()
    rp = torch.as_tensor(rp.astype(np.int64), device="cuda")
    ci = torch.as_tensor(ci.astype(np.int64), device="cuda")
    Nt = torch.sparse_csr_tensor(rp, ci, nval, size=(m, m))
    x = torch.randn(m, dtype=torch.float64, device="cuda")
    y = (Nt @ x.unsqueeze(1)).squeeze(1)
    t = torch.empty(n, dtype=torch.float64, device="cuda")
    A.spmv(x, t, trans=1)
    t *= D
    z = torch.empty(m, dtype=torch.float64, device="cuda")
    A.spmv(t, z, trans=0)
    z += dyn * x
    err = (y - z).abs().max().item()
    scale = (Nt.abs() @ x.abs().unsqueeze(1)).abs().max().item()
    assert err <= 1e-12 * scale * 10
    # symmetry of the pattern: nnz per row equals nnz per column
    row_cnt = torch.diff(rp)
    col_cnt = torch.bincount(ci, minlength=m)
    assert torch.equal(row_cnt, col_cnt)


def test_large_zipf_sampled_rows_match_oracle(hn, torch_cuda):
    """The benchmarked size (m 200k, n 500k, 5.16M nonzeros, nnz(N) 9.7e8):
    4,096 rows of N -- the 64 longest and a seeded sample of the rest --
    against the row-restricted oracle restatement of build_normal_equations.
    Pattern bit-exact, values within 1e-12 normwise, dyn_reg equal."""
    import ctypes as C

    torch = torch_cuda
    lp = lpgen.scaled_problem(lpgen.lp_zipf(seed=1000))
    m, n = lp["m"], lp["n"]
    A = hn.Csr(m, n, lp["rp"], lp["ci"], lp["val"])
    P = hn.Pattern(A)
    D = np.random.default_rng(17).uniform(0.5, 1.5, n)
    nval = torch.empty(P.nnz, dtype=torch.float64, device="cuda")
    dyn = torch.empty(1, dtype=torch.float64, device="cuda")
    P.numeric(torch.as_tensor(D, device="cuda"), 1e-8, nval, dyn)
    torch.cuda.synchronize()
    rp_d, ci_d, _ = P.device_arrays()
    lib = hn.load()
    rpN = np.empty(m + 1, dtype=np.int64)
    hn.check(lib.hn_memcpy_d2h(rpN.ctypes.data, rp_d, 8 * (m + 1), None))
    lens = np.diff(rpN)
    longest = np.argsort(-lens, kind="stable")[:64]
    rest = np.setdiff1d(np.arange(m), longest)
    rows = np.sort(np.concatenate([longest, np.random.default_rng(5).choice(rest, 4096 - 64, replace=False)]))
    rpS, ciS, vS, aS, dynS = O.normal_rows(lp["rp"], lp["ci"], lp["val"], D, 1e-8, n, rows)
    assert float(dyn.item()) == dynS
    for s, i in enumerate(rows):
        a, b = int(rpN[i]), int(rpN[i + 1])
        assert b - a == rpS[s + 1] - rpS[s], (i, b - a, rpS[s + 1] - rpS[s])
        cols = np.empty(b - a, dtype=np.int32)
        hn.check(lib.hn_memcpy_d2h(cols.ctypes.data, C.c_void_p(ci_d + 4 * a), 4 * (b - a), None))
        assert np.array_equal(cols.astype(np.int64), ciS[rpS[s]:rpS[s + 1]]), i
        got = nval[a:b].cpu().numpy()
        ref, scale = vS[rpS[s]:rpS[s + 1]], aS[rpS[s]:rpS[s + 1]]
        assert np.all(np.abs(got - ref) <= 1e-12 * scale), (i, np.max(np.abs(got - ref) / scale))


@pytest.mark.parametrize("shape", [(2000, 5000, 8, 0), (529, 1322, 6, 7), (3000, 6000, 40, 3)])
def test_numeric_layouts_bit_identical(hn, torch_cuda, shape):
    """The three numeric layouts (row mode, gather mode, relative map) give
    the same bits, with inactive columns (d_j = 0) and three or more terms in
    some slots; the last shape has rows of N of ~1,300 slots on average."""
    m, n, k, seed = shape
    lp = lpgen.scaled_problem(lpgen.lp_uniform(m, n, k, seed))
    D = np.random.default_rng(seed).uniform(1e-3, 1e3, n)
    D[::17] = 0.0  # inactive columns
    A = hn.Csr(m, n, lp["rp"], lp["ci"], lp["val"])
    Dd = torch_cuda.as_tensor(D, device="cuda")
    out = []
    for layout in (hn.Pattern.ROW, hn.Pattern.GATHER, hn.Pattern.RELATIVE):
        P = hn.Pattern(A, layout=layout)
        assert P.mode()[0] == layout
        nval = torch_cuda.empty(P.nnz, dtype=torch_cuda.float64, device="cuda")
        dyn = torch_cuda.empty(1, dtype=torch_cuda.float64, device="cuda")
        P.numeric(Dd, 1e-8, nval, dyn)
        torch_cuda.cuda.synchronize()
        out.append((P.export(), nval.cpu().numpy(), dyn.item()))
    (p0, v0, d0) = out[0]
    for (p1, v1, d1) in out[1:]:
        assert np.array_equal(p0[0], p1[0]) and np.array_equal(p0[1], p1[1])
        assert np.array_equal(v0, v1) and d0 == d1
    # the library's choice: the relative map for rows of N of >= 2,048 slots on average
    P = hn.Pattern(A)
    assert P.mode()[0] == (hn.Pattern.RELATIVE if P.nnz >= 2048 * m else hn.Pattern.GATHER)
    check_values(lp, D, 1e-8, p0[0].astype(np.int64), p0[1].astype(np.int64), v0, d0)


def test_long_row_of_a_selects_gather_mode(hn, torch_cuda):
    """A row of A with more than 256 entries: gather mode even when row mode
    is asked for, values still match build_normal_equations."""
    m, n = 300, 1500
    lp = lpgen.scaled_problem(lpgen.lp_uniform(m, n, 4, 21))
    rows = [lp["ci"][lp["rp"][i]:lp["rp"][i + 1]] for i in range(m)]
    vals = [lp["val"][lp["rp"][i]:lp["rp"][i + 1]] for i in range(m)]
    dense = np.arange(0, n, 2)  # 750 entries in row 0
    rows[0] = dense
    vals[0] = np.random.default_rng(2).uniform(0.1, 1.0, dense.size)
    rp = np.concatenate([[0], np.cumsum([r.size for r in rows])]).astype(np.int64)
    lp2 = dict(lp, rp=rp, ci=np.concatenate(rows).astype(np.int64), val=np.concatenate(vals))
    D = np.random.default_rng(5).uniform(0.1, 10, n)
    A, P, rp_, ci_, vals_, dyn = assemble(hn, torch_cuda, lp2, D, compact=True)
    assert P.mode()[0] != hn.Pattern.ROW
    check_values(lp2, D, 1e-8, rp_, ci_, vals_, dyn)
    # the relative map stages a row's entries in a 256-entry slice: not taken either
    assert hn.Pattern(A, layout=hn.Pattern.RELATIVE).mode()[0] == hn.Pattern.GATHER


def test_row_layout_long_rows_bit_identical_to_gather(hn, torch_cuda):
    """Rows of N longer than the row layout's 8,192-slot shared-memory window
    (m 30,000, n 90,000, 60 nonzeros per column: ~9,000 slots per row, rows of
    A 180 entries on average, 236 at most): the row layout assembles each row
    in several windows, the relative map stages rows of A of up to 236
    entries in its warp's shared slice, and both
    must give the gather layout's bits (the gather layout is pinned to the
    oracle by the tests above)."""
    torch = torch_cuda
    lp = lpgen.scaled_problem(lpgen.lp_uniform(30000, 90000, 60, 5))
    m, n = lp["m"], lp["n"]
    D = np.random.default_rng(8).uniform(1e-3, 1e3, n)
    D[::29] = 0.0
    A = hn.Csr(m, n, lp["rp"], lp["ci"], lp["val"])
    Dd = torch.as_tensor(D, device="cuda")
    out = []
    for layout in (hn.Pattern.ROW, hn.Pattern.GATHER, hn.Pattern.RELATIVE):
        P = hn.Pattern(A, layout=layout)
        assert P.mode()[0] == layout
        if layout == hn.Pattern.ROW:
            assert P.mode()[1] > 8192
        nval = torch.empty(P.nnz, dtype=torch.float64, device="cuda")
        dyn = torch.empty(1, dtype=torch.float64, device="cuda")
        P.numeric(Dd, 1e-8, nval, dyn)
        torch.cuda.synchronize()
        out.append((nval.cpu().numpy(), dyn.item()))
        del P, nval
    for v, d in out[1:]:
        assert np.array_equal(out[0][0], v) and out[0][1] == d
