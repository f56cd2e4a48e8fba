"""GPU: the GNN warm-start kernels (hn_gnn_*) against the numpy oracle
(oracle/gnn_oracle.py, same BF16 operand rounding, float64 accumulation),
training on the GPU, and the trained network's prediction used as an IPM
warm start (same status and objective as the cold solve, 1e-8)."""
import numpy as np
import pytest

import gnn
import gnn_oracle as GO
import lpgen

pytestmark = pytest.mark.gpu


def rel_norm(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


def batch_and_net(torch, lps, seed=0):
    rng = np.random.default_rng(seed)
    sols = [(rng.uniform(0, 2, lp["n"]), rng.standard_normal(lp["m"]), rng.uniform(0, 1, lp["n"])) for lp in lps]
    B = gnn.Batch(lps, sols)
    model = gnn.Model(seed=seed)
    rp, ci, m_off, n_off = gnn.pack(lps)
    vr, vc = zip(*(gnn.normalised_values(lp) for lp in lps))
    Ar = GO.csr_dense(B.m, B.n, rp, ci, np.concatenate(vr))
    Ac = GO.csr_dense(B.m, B.n, rp, ci, np.concatenate(vc))
    net = GO.Net(gnn.layer_shapes(), model.params().astype(np.float64), Ar, Ac, B.Fv.cpu().numpy(),
                 B.Fc.cpu().numpy(), bf16=True)
    return B, model, net


def test_forward_and_gradients_match_oracle(hn, torch_cuda):
    lps = [lpgen.lp_uniform(60, 150, 6, 1), lpgen.lp_uniform(90, 225, 6, 2), lpgen.lp_uniform(35, 88, 6, 3)]
    B, model, net = batch_and_net(torch_cuda, lps)
    cache = gnn.forward(model, B)
    ref = net.forward()
    for k in ("ov", "oc"):
        assert rel_norm(cache[k].cpu().numpy().astype(np.float64), ref[k]) <= 1e-2, k
    for l in range(gnn.LAYERS + 1):
        assert rel_norm(cache["hv"][l].cpu().numpy().astype(np.float64), ref["hv"][l]) <= 1e-2
        assert rel_norm(cache["hc"][l].cpu().numpy().astype(np.float64), ref["hc"][l]) <= 1e-2
    loss = gnn.backward(model, B, cache)
    Tv, Tc = B.Tv.cpu().numpy().astype(np.float64), B.Tc.cpu().numpy().astype(np.float64)
    assert abs(loss - net.loss(Tv, Tc)) <= 1e-3 * abs(net.loss(Tv, Tc))
    g_ref = net.backward(Tv, Tc)
    g = model.g.cpu().numpy().astype(np.float64)
    offs, _ = gnn.param_offsets()
    for name, (o, K) in offs.items():
        w = slice(o, o + K * 64)
        b = slice(o + K * 64, o + K * 64 + 64)
        assert rel_norm(g[w], g_ref[w]) <= 3e-2, (name, rel_norm(g[w], g_ref[w]))
        assert rel_norm(g[b], g_ref[b]) <= 3e-2, (name, rel_norm(g[b], g_ref[b]))


def test_backward_is_deterministic(hn, torch_cuda):
    lps = [lpgen.lp_uniform(200, 500, 6, 7)]
    B, model, _ = batch_and_net(torch_cuda, lps)
    out = []
    for _ in range(2):
        cache = gnn.forward(model, B)
        gnn.backward(model, B, cache)
        out.append(model.g.cpu().numpy().copy())
    assert np.array_equal(out[0], out[1])


def test_training_lowers_the_loss_and_warm_start_keeps_the_answer(hn, torch_cuda):
    """Train on IPM solutions of small C0-generator LPs; the prediction for
    held-out LPs warm-starts the IPM without changing status or objective,
    and saves iterations: the held-out mean drops by at least one (measured
    16.6 -> 12.8; everything here is seeded and the kernels deterministic)."""
    sizes = [int(v) for v in np.exp(np.random.default_rng(0).uniform(np.log(60), np.log(200), 40))]
    lps = [lpgen.lp_uniform(m, int(round(2.5 * m)), 8, 50000 + i) for i, m in enumerate(sizes)]
    r = hn.lp_solve_batch(lps)
    assert np.all(r["status"] == 1)
    sols = []
    for k, lp in enumerate(lps):
        c0, c1 = r["col_off"][k], r["col_off"][k + 1]
        r0, r1 = r["row_off"][k], r["row_off"][k + 1]
        sols.append((r["x"][c0:c1], r["y"][r0:r1], r["s"][c0:c1]))
    train, held = list(range(32)), list(range(32, 40))
    batches = [gnn.Batch([lps[i] for i in train[j:j + 8]], [sols[i] for i in train[j:j + 8]])
               for j in range(0, 32, 8)]
    model = gnn.Model(seed=1)
    losses = gnn.train(model, batches, epochs=40, lr=2e-3)
    assert losses[-1] < 0.5 * losses[0], losses[::10]
    Bh = gnn.Batch([lps[i] for i in held])
    preds = gnn.predict(model, Bh)
    used, it_warm, it_cold = 0, [], []
    for k, i in enumerate(held):
        x, y, s = preds[k]
        w = hn.lp_solve(lps[i], x0=x, y0=y, s0=s, warm_floor=gnn.WARM_FLOOR)
        cold = hn.lp_solve(lps[i])
        used += int(w["warm_start_used"])
        it_warm.append(w["iterations"])
        it_cold.append(cold["iterations"])
        assert w["status"] == cold["status"] == 1
        assert abs(w["objective"] - cold["objective"]) <= 1e-8 * (1 + abs(cold["objective"]))
    assert used == len(held)
    assert np.mean(it_warm) <= np.mean(it_cold) - 1.0, (it_warm, it_cold)


@pytest.mark.parametrize("K1,K2,relu,M", [(16, 0, 1, 1000), (64, 64, 1, 4097), (64, 0, 0, 130), (32, 32, 1, 128),
                                            (64, 64, 1, 148 * 128 * 3 + 77), (16, 0, 0, 40000), (48, 16, 1, 20001)])
def test_tcgen05_layer_matches_mma_sync_layer(hn, torch_cuda, K1, K2, relu, M):
    """hn_gnn_linear_umma (tcgen05, TMEM accumulator) against hn_gnn_linear
    (mma.sync): same BF16 operands, FP32 accumulation in a different order.
    The larger cases give every persistent CTA several tiles (both staging
    buffers cycle more than once) and end on a partial tile."""
    torch = torch_cuda
    g = torch.Generator(device="cuda").manual_seed(K1 + K2 + M)
    X1 = torch.randn((M, K1), generator=g, device="cuda")
    X2 = torch.randn((M, K2), generator=g, device="cuda") if K2 else None
    K = K1 + K2
    W = torch.randn(K * 64, generator=g, device="cuda") / K ** 0.5
    b = torch.randn(64, generator=g, device="cuda")
    Wt = torch.empty(K * 64, dtype=torch.bfloat16, device="cuda")
    Wb = torch.empty(K * 64, dtype=torch.bfloat16, device="cuda")
    lib = hn.load()
    hn.check(lib.hn_gnn_cast_weights(K, W.data_ptr(), Wt.data_ptr(), Wb.data_ptr(), None))
    ys = []
    for fn in ("mma", "umma"):
        Y = torch.full((M, 64), float("nan"), device="cuda")
        x2 = None if X2 is None else X2.data_ptr()
        if fn == "mma":
            hn.check(lib.hn_gnn_linear(M, K1, K2, X1.data_ptr(), x2, Wt.data_ptr(), 64, b.data_ptr(), relu,
                                       Y.data_ptr(), None))
        else:
            hn.check(lib.hn_gnn_linear_umma(M, K1, K2, X1.data_ptr(), x2, Wt.data_ptr(), b.data_ptr(), relu,
                                            Y.data_ptr(), None))
            hn.check(lib.hn_gnn_check(None))
        torch.cuda.synchronize()
        ys.append(Y.cpu().numpy().astype(np.float64))
    assert np.all(np.isfinite(ys[1]))
    scale = np.abs(ys[0]).max() + 1.0
    assert np.max(np.abs(ys[1] - ys[0])) <= 1e-5 * scale


@pytest.mark.parametrize("polls", [1, 8])
def test_tcgen05_wait_timeout_is_reported_and_the_context_recovers(hn, torch_cuda, polls):
    """The tcgen05 layer's pipeline waits are bounded. With the test hook's
    limit of a few polls, the first waits give up while the CTA's own bulk
    copies are still in flight: the kernel records the timeout, settles those
    copies (and any MMA it issued) with the full bound, frees TMEM and
    returns; hn_gnn_check reports the error and clears it. Afterwards the
    same call with the normal limit succeeds and matches the mma.sync layer:
    nothing hung, nothing faulted, the context is usable."""
    torch = torch_cuda
    M, K1, K2 = 148 * 128 * 2 + 5, 64, 64
    g = torch.Generator(device="cuda").manual_seed(7)
    X1 = torch.randn((M, K1), generator=g, device="cuda")
    X2 = torch.randn((M, K2), generator=g, device="cuda")
    W = torch.randn(128 * 64, generator=g, device="cuda") / 128 ** 0.5
    b = torch.randn(64, generator=g, device="cuda")
    Wt = torch.empty(128 * 64, dtype=torch.bfloat16, device="cuda")
    Wb = torch.empty(128 * 64, dtype=torch.bfloat16, device="cuda")
    lib = hn.load()
    hn.check(lib.hn_gnn_cast_weights(128, W.data_ptr(), Wt.data_ptr(), Wb.data_ptr(), None))
    Y = torch.empty((M, 64), device="cuda")
    hn.check(lib.hn_gnn_check(None))  # no stale flag
    try:
        hn.check(lib.hn_gnn_set_wait_limit(polls))
        hn.check(lib.hn_gnn_linear_umma(M, K1, K2, X1.data_ptr(), X2.data_ptr(), Wt.data_ptr(), b.data_ptr(), 1,
                                        Y.data_ptr(), None))
        st = lib.hn_gnn_check(None)
        assert st == hn.HN_ERR_CUDA, st
        assert b"timed out" in lib.hn_last_error()
    finally:
        hn.check(lib.hn_gnn_set_wait_limit(0))
    assert lib.hn_gnn_check(None) == hn.HN_OK  # the flag was cleared
    ref = torch.empty((M, 64), device="cuda")
    hn.check(lib.hn_gnn_linear(M, K1, K2, X1.data_ptr(), X2.data_ptr(), Wt.data_ptr(), 64, b.data_ptr(), 1,
                               ref.data_ptr(), None))
    hn.check(lib.hn_gnn_linear_umma(M, K1, K2, X1.data_ptr(), X2.data_ptr(), Wt.data_ptr(), b.data_ptr(), 1,
                                    Y.data_ptr(), None))
    hn.check(lib.hn_gnn_check(None))
    torch.cuda.synchronize()
    y, r = Y.cpu().numpy().astype(np.float64), ref.cpu().numpy().astype(np.float64)
    assert np.max(np.abs(y - r)) <= 1e-5 * (np.abs(r).max() + 1.0)


def _bf16(torch, t):
    return t.to(torch.bfloat16).to(torch.float64).cpu().numpy()


def _linear_bwd(hn, torch, lib, M, K1, K2, relu, X1, X2, Wb, Y, dY, with_dx):
    K = K1 + K2
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    nb = max(1, min((M + 63) // 64, sms))
    scratch = torch.empty(nb * (64 * K + 64), device="cuda")
    G = torch.empty((M, 64), device="cuda")
    dX = torch.full((M, K), float("nan"), device="cuda") if with_dx else None
    dW = torch.full((K, 64), float("nan"), device="cuda")
    db = torch.full((64,), float("nan"), device="cuda")
    hn.check(lib.hn_gnn_linear_bwd(M, K1, K2, X1.data_ptr(), None if X2 is None else X2.data_ptr(), Wb.data_ptr(),
                                   Y.data_ptr(), dY.data_ptr(), relu, G.data_ptr(),
                                   None if dX is None else dX.data_ptr(), dW.data_ptr(), db.data_ptr(),
                                   scratch.data_ptr(), scratch.numel(), None))
    return G, dX, dW, db


@pytest.mark.parametrize("K1,K2,relu,M", [(16, 0, 1, 1000), (64, 0, 0, 130), (64, 64, 1, 4097), (32, 32, 1, 64),
                                            (64, 64, 1, 148 * 64 * 3 + 77), (48, 16, 0, 20001), (16, 0, 1, 1),
                                            (64, 64, 0, 148 * 128 * 2 + 5)])
def test_tcgen05_backward_matches_float64_of_the_bf16_operands(hn, torch_cuda, K1, K2, relu, M):
    """hn_gnn_linear_bwd: dX = G W^T (the tcgen05 layer kernel with 64 or 128
    outputs) and dW = [X1 | X2]^T G (the tcgen05 weight-gradient kernel, one
    TMEM accumulator per persistent CTA over its 64-row tiles) against a
    float64 product of the same BF16-rounded operands; db against the FP32
    G. Every element is within 1e-4 of the sum of its terms' magnitudes
    (FP32 accumulation; a wrong operand layout or a dropped tile gives errors
    of order one). The larger cases give each CTA several tiles (all three
    staging buffers cycle) and end on a partial tile; M = 1 is one row."""
    torch = torch_cuda
    g = torch.Generator(device="cuda").manual_seed(K1 * 7 + K2 + M)
    K = K1 + K2
    X1 = torch.randn((M, K1), generator=g, device="cuda")
    X2 = torch.randn((M, K2), generator=g, device="cuda") if K2 else None
    W = torch.randn(K * 64, generator=g, device="cuda") / K ** 0.5
    Wt = torch.empty(K * 64, dtype=torch.bfloat16, device="cuda")
    Wb = torch.empty(K * 64, dtype=torch.bfloat16, device="cuda")
    Y = torch.randn((M, 64), generator=g, device="cuda")
    dY = torch.randn((M, 64), generator=g, device="cuda")
    lib = hn.load()
    hn.check(lib.hn_gnn_cast_weights(K, W.data_ptr(), Wt.data_ptr(), Wb.data_ptr(), None))
    with_dx = K in (64, 128)
    G, dX, dW, db = _linear_bwd(hn, torch, lib, M, K1, K2, relu, X1, X2, Wb, Y, dY, with_dx)
    hn.check(lib.hn_gnn_check(None))
    torch.cuda.synchronize()
    Gf = torch.where(Y > 0, dY, torch.zeros_like(dY)) if relu else dY
    assert torch.equal(G, Gf)
    Gb = _bf16(torch, Gf)
    X = X1 if X2 is None else torch.cat([X1, X2], dim=1)
    Xb = _bf16(torch, X)
    Wd = _bf16(torch, W.view(K, 64))
    dW_ref = Xb.T @ Gb
    bound = 1e-4 * (np.abs(Xb).T @ np.abs(Gb)) + 1e-30
    assert np.all(np.abs(dW.cpu().numpy().astype(np.float64) - dW_ref) <= bound)
    Gd = Gf.to(torch.float64).cpu().numpy()
    assert np.all(np.abs(db.cpu().numpy() - Gd.sum(0)) <= 1e-4 * np.abs(Gd).sum(0) + 1e-30)
    if with_dx:
        dX_ref = Gb @ Wd.T
        bx = 1e-4 * (np.abs(Gb) @ np.abs(Wd).T) + 1e-30
        assert np.all(np.abs(dX.cpu().numpy().astype(np.float64) - dX_ref) <= bx)
    # deterministic: a second call gives the same bits
    _, dX2, dW2, db2 = _linear_bwd(hn, torch, lib, M, K1, K2, relu, X1, X2, Wb, Y, dY, with_dx)
    assert torch.equal(dW, dW2) and torch.equal(db, db2)
    assert (not with_dx) or torch.equal(dX, dX2)


@pytest.mark.parametrize("polls", [1, 8])
def test_tcgen05_backward_wait_timeout_is_reported_and_the_context_recovers(hn, torch_cuda, polls):
    """The backward's tcgen05 kernels (dX and dW) share the layer's bounded
    waits and flag: with the test hook's few polls they give up while their
    own bulk copies are in flight, settle them with the full bound, free
    TMEM and return; hn_gnn_check reports it. Then the normal limit gives
    the same result as a fresh run."""
    torch = torch_cuda
    M, K1, K2 = 148 * 128 * 2 + 5, 64, 64
    g = torch.Generator(device="cuda").manual_seed(11)
    X1 = torch.randn((M, K1), generator=g, device="cuda")
    X2 = torch.randn((M, K2), generator=g, device="cuda")
    W = torch.randn(128 * 64, generator=g, device="cuda") / 128 ** 0.5
    Wt = torch.empty(128 * 64, dtype=torch.bfloat16, device="cuda")
    Wb = torch.empty(128 * 64, dtype=torch.bfloat16, device="cuda")
    Y = torch.randn((M, 64), generator=g, device="cuda")
    dY = torch.randn((M, 64), generator=g, device="cuda")
    lib = hn.load()
    hn.check(lib.hn_gnn_cast_weights(128, W.data_ptr(), Wt.data_ptr(), Wb.data_ptr(), None))
    ref = _linear_bwd(hn, torch, lib, M, K1, K2, 1, X1, X2, Wb, Y, dY, True)
    hn.check(lib.hn_gnn_check(None))
    try:
        hn.check(lib.hn_gnn_set_wait_limit(polls))
        _linear_bwd(hn, torch, lib, M, K1, K2, 1, X1, X2, Wb, Y, dY, True)
        st = lib.hn_gnn_check(None)
        assert st == hn.HN_ERR_CUDA, st
        assert b"timed out" in lib.hn_last_error()
    finally:
        hn.check(lib.hn_gnn_set_wait_limit(0))
    assert lib.hn_gnn_check(None) == hn.HN_OK
    out = _linear_bwd(hn, torch, lib, M, K1, K2, 1, X1, X2, Wb, Y, dY, True)
    hn.check(lib.hn_gnn_check(None))
    for a, b in zip(ref, out):
        assert torch.equal(a, b)
