"""GNN warm start for the IPM (no counterpart in the reference, whose IPM
always starts from Mehrotra's default point, core/lp/interior_point.cpp:443-453).

A bipartite variable-constraint network over the LP's matrix A:

    h_v = relu(F_v W_ev + b),  h_c = relu(F_c W_ec + b)             (embed, 16 -> 64)
    for l in 0..3:
        h_c = relu([h_c | A_r h_v] W_c[l] + b)                        (128 -> 64)
        h_v = relu([h_v | A_c^T h_c] W_v[l] + b)                      (128 -> 64)
    o_v = h_v W_hv + b,  o_c = h_c W_hc + b                           (heads)

A_r = diag(1/row degree) A and A_c = A diag(1/column degree) (mean
aggregation). The heads predict log1p(x*), log1p(s*) per variable and y* per
constraint; the IPM takes x = expm1(max(o, 0)), s likewise, y = o_c as a warm
start (hnb200.lp_solve(..., x0, y0, s0)), which it shifts to strict interiority
and keeps only when its KKT residual beats the default start.

Every step runs on the sm_100a library (include/hn_sm100.h, hn_gnn_*):
aggregations are its 64-wide SpMM over the device A and A^T, the forward
layers are BF16 tcgen05 MMAs with FP32 accumulation in tensor memory, the
backward's GEMMs BF16 mma.sync tiles, and Adam updates FP32 master weights. PyTorch only holds the device
buffers.
"""
from __future__ import annotations

import numpy as np

import hnb200 as hn

H = 64
FEAT = 16
LAYERS = 4
# shift floor for the IPM's warm start from a prediction (hnb200.lp_solve's
# warm_floor): chosen on held-out LPs of m 60-400 (mean iterations 19.4 cold,
# 15.7 at 0.01, 14.8 at 0.05, 16.4 at 0.2)
WARM_FLOOR = 0.05


# ---------------------------------------------------------------- host-side data
def features(lp: dict):
    """Variable and constraint input features (n x 16, m x 16, float32)."""
    m, n = int(lp["m"]), int(lp["n"])
    rp = np.asarray(lp["rp"], np.int64)
    ci = np.asarray(lp["ci"], np.int64)
    val = np.asarray(lp["val"], np.float64)
    b, c = np.asarray(lp["b"], np.float64), np.asarray(lp["c"], np.float64)
    deg_r = np.diff(rp).astype(np.float64)
    rows = np.repeat(np.arange(m), np.diff(rp))
    rowabs = np.bincount(rows, weights=np.abs(val), minlength=m)
    deg_c = np.bincount(ci, minlength=n).astype(np.float64)
    colabs = np.bincount(ci, weights=np.abs(val), minlength=n)
    cmax = max(np.max(np.abs(c)), 1e-30) if n else 1.0
    bmax = max(np.max(np.abs(b)), 1e-30) if m else 1.0
    Fv = np.zeros((n, FEAT), np.float32)
    Fv[:, 0] = c / cmax
    Fv[:, 1] = c / np.maximum(colabs, 1e-30)
    Fv[:, 2] = deg_c / 10.0
    Fv[:, 3] = colabs / np.maximum(deg_c, 1.0)
    Fv[:, 4] = 1.0
    Fc = np.zeros((m, FEAT), np.float32)
    Fc[:, 0] = b / bmax
    Fc[:, 1] = b / np.maximum(rowabs, 1e-30)
    Fc[:, 2] = deg_r / 20.0
    Fc[:, 3] = rowabs / np.maximum(deg_r, 1.0)
    Fc[:, 4] = 1.0
    return Fv, Fc


def targets(x, y, s):
    """Per-variable (log1p x, log1p s) and per-constraint (y, 0), float32."""
    Tv = np.stack([np.log1p(np.maximum(x, 0.0)), np.log1p(np.maximum(s, 0.0))], 1).astype(np.float32)
    Tc = np.stack([y, np.zeros_like(y)], 1).astype(np.float32)
    return Tv, Tc


def normalised_values(lp: dict):
    """Values of A_r = diag(1/row deg) A and A_c = A diag(1/col deg)."""
    rp = np.asarray(lp["rp"], np.int64)
    ci = np.asarray(lp["ci"], np.int64)
    val = np.asarray(lp["val"], np.float64)
    deg_r = np.maximum(np.diff(rp), 1).astype(np.float64)
    deg_c = np.maximum(np.bincount(ci, minlength=int(lp["n"])), 1).astype(np.float64)
    rows = np.repeat(np.arange(int(lp["m"])), np.diff(rp))
    return val / deg_r[rows], val / deg_c[ci]


def layer_shapes():
    """(name, fan-in) of every layer, in the order of the flat parameter buffer."""
    shapes = [("ev", FEAT), ("ec", FEAT)]
    for l in range(LAYERS):
        shapes += [(f"c{l}", 2 * H), (f"v{l}", 2 * H)]
    shapes += [("hv", H), ("hc", H)]
    return shapes


def init_params(seed: int = 0) -> np.ndarray:
    """Flat FP32 parameters: per layer W (K x 64, row-major) then b (64)."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, K in layer_shapes():
        std = np.sqrt((1.0 if name in ("hv", "hc") else 2.0) / K)
        parts.append(rng.normal(0.0, std, size=K * H))
        parts.append(np.zeros(H))
    return np.concatenate(parts).astype(np.float32)


def param_offsets():
    off, out = 0, {}
    for name, K in layer_shapes():
        out[name] = (off, K)
        off += K * H + H
    return out, off


def pack(lps: list):
    """Block-diagonal packing of several LPs (CSR arrays, offsets)."""
    m_off = np.cumsum([0] + [int(lp["m"]) for lp in lps])
    n_off = np.cumsum([0] + [int(lp["n"]) for lp in lps])
    rps, cis, nnz = [], [], 0
    for k, lp in enumerate(lps):
        rp = np.asarray(lp["rp"], np.int64)
        rps.append(rp[(1 if k else 0):] + nnz)
        cis.append(np.asarray(lp["ci"], np.int64) + n_off[k])
        nnz += int(rp[-1])
    return np.concatenate(rps), np.concatenate(cis), m_off, n_off


# ---------------------------------------------------------------- device model
class Model:
    """FP32 master weights, their BF16 copies, Adam state (device)."""

    def __init__(self, params: np.ndarray | None = None, seed: int = 0):
        import torch

        self.torch = torch
        self.offsets, self.size = param_offsets()
        p = init_params(seed) if params is None else np.asarray(params, np.float32)
        assert p.size == self.size
        self.w = torch.as_tensor(p.copy(), device="cuda")
        self.g = torch.zeros_like(self.w)
        self.m1 = torch.zeros_like(self.w)
        self.m2 = torch.zeros_like(self.w)
        self.step_count = 0
        self.wt = {}
        self.wb = {}
        for name, K in layer_shapes():
            self.wt[name] = torch.empty(K * H, dtype=torch.bfloat16, device="cuda")
            self.wb[name] = torch.empty(K * H, dtype=torch.bfloat16, device="cuda")
        self.cast()

    def W(self, name):
        o, K = self.offsets[name]
        return self.w[o:o + K * H]

    def b(self, name):
        o, K = self.offsets[name]
        return self.w[o + K * H:o + K * H + H]

    def dW(self, name):
        o, K = self.offsets[name]
        return self.g[o:o + K * H]

    def db(self, name):
        o, K = self.offsets[name]
        return self.g[o + K * H:o + K * H + H]

    def cast(self):
        lib = hn.load()
        for name, K in layer_shapes():
            hn.check(lib.hn_gnn_cast_weights(K, self.W(name).data_ptr(), self.wt[name].data_ptr(),
                                             self.wb[name].data_ptr(), None))

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step_count += 1
        hn.check(hn.load().hn_gnn_adam(self.size, self.w.data_ptr(), self.g.data_ptr(), self.m1.data_ptr(),
                                       self.m2.data_ptr(), lr, beta1, beta2, eps, self.step_count, None))
        self.cast()

    def params(self) -> np.ndarray:
        return self.w.cpu().numpy()


class Batch:
    """Several LPs packed block-diagonally, with features (and targets)."""

    def __init__(self, lps: list, sols: list | None = None):
        import torch

        self.lps = lps
        rp, ci, self.m_off, self.n_off = pack(lps)
        self.m, self.n = int(self.m_off[-1]), int(self.n_off[-1])
        vr, vc = zip(*(normalised_values(lp) for lp in lps))
        # the aggregations use the SpMM kernel, not the SpMV paths: no autotuning
        self.Ar = hn.Csr(self.m, self.n, rp, ci, np.concatenate(vr), autotune=False)
        self.Ac = hn.Csr(self.m, self.n, rp, ci, np.concatenate(vc), autotune=False)
        F = [features(lp) for lp in lps]
        dev = "cuda"
        self.Fv = torch.as_tensor(np.concatenate([f[0] for f in F]), device=dev)
        self.Fc = torch.as_tensor(np.concatenate([f[1] for f in F]), device=dev)
        self.Tv = self.Tc = None
        if sols is not None:
            T = [targets(*s) for s in sols]
            self.Tv = torch.as_tensor(np.concatenate([t[0] for t in T]), device=dev)
            self.Tc = torch.as_tensor(np.concatenate([t[1] for t in T]), device=dev)


def _empty(torch, rows, cols=H):
    return torch.empty((rows, cols), dtype=torch.float32, device="cuda")


def forward(model: Model, B: Batch):
    """Returns the cache: activations of every layer and the two head outputs."""
    torch = model.torch
    lib = hn.load()

    def lin(X1, X2, name, relu, rows):
        # the layers run on the tcgen05 tensor cores (hn_gnn_linear_umma)
        K1 = X1.shape[1]
        K2 = 0 if X2 is None else X2.shape[1]
        Y = _empty(torch, rows)
        hn.check(lib.hn_gnn_linear_umma(rows, K1, K2, X1.data_ptr(), None if X2 is None else X2.data_ptr(),
                                        model.wt[name].data_ptr(), model.b(name).data_ptr(), relu, Y.data_ptr(),
                                        None))
        return Y

    hv = [lin(B.Fv, None, "ev", 1, B.n)]
    hc = [lin(B.Fc, None, "ec", 1, B.m)]
    ac, av = [], []
    for l in range(LAYERS):
        a = _empty(torch, B.m)
        hn.check(lib.hn_gnn_spmm(B.Ar.h, 0, hv[-1].data_ptr(), a.data_ptr(), 0, None))
        ac.append(a)
        hc.append(lin(hc[-1], a, f"c{l}", 1, B.m))
        a = _empty(torch, B.n)
        hn.check(lib.hn_gnn_spmm(B.Ac.h, 1, hc[-1].data_ptr(), a.data_ptr(), 0, None))
        av.append(a)
        hv.append(lin(hv[-1], a, f"v{l}", 1, B.n))
    ov = lin(hv[-1], None, "hv", 0, B.n)
    oc = lin(hc[-1], None, "hc", 0, B.m)
    hn.check(lib.hn_gnn_check(None))
    return {"hv": hv, "hc": hc, "ac": ac, "av": av, "ov": ov, "oc": oc}


def backward(model: Model, B: Batch, cache: dict):
    """Fills model.g with the gradient of the mean squared error of the heads
    (variables: mean over n of both columns; constraints: mean over m);
    returns the loss."""
    torch = model.torch
    lib = hn.load()
    nparts = 1024
    lp_v = torch.zeros(nparts, dtype=torch.float32, device="cuda")
    lp_c = torch.zeros(nparts, dtype=torch.float32, device="cuda")
    dov, doc = _empty(torch, B.n), _empty(torch, B.m)
    hn.check(lib.hn_gnn_head_grad(B.n, cache["ov"].data_ptr(), B.Tv.data_ptr(), 2, 1.0 / B.n, dov.data_ptr(),
                                  lp_v.data_ptr(), nparts, None))
    hn.check(lib.hn_gnn_head_grad(B.m, cache["oc"].data_ptr(), B.Tc.data_ptr(), 1, 1.0 / B.m, doc.data_ptr(),
                                  lp_c.data_ptr(), nparts, None))
    rows_max = max(B.n, B.m)
    # one dW/db partial per CTA of the weight-gradient kernel (at most one per SM)
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    scratch_len = max(1, min((rows_max + 63) // 64, sms)) * (H * 2 * H + H)
    scratch = torch.empty(scratch_len, dtype=torch.float32, device="cuda")
    G = torch.empty(rows_max * H, dtype=torch.float32, device="cuda")

    def lin_bwd(X1, X2, name, Y, dY, relu, rows, dX):
        K1 = X1.shape[1]
        K2 = 0 if X2 is None else X2.shape[1]
        hn.check(lib.hn_gnn_linear_bwd(rows, K1, K2, X1.data_ptr(), None if X2 is None else X2.data_ptr(),
                                       model.wb[name].data_ptr(), Y.data_ptr(), dY.data_ptr(), relu, G.data_ptr(),
                                       None if dX is None else dX.data_ptr(), model.dW(name).data_ptr(),
                                       model.db(name).data_ptr(), scratch.data_ptr(), scratch_len, None))

    hv, hc, ac, av = cache["hv"], cache["hc"], cache["ac"], cache["av"]
    dhv, dhc = _empty(torch, B.n), _empty(torch, B.m)
    lin_bwd(hv[-1], None, "hv", cache["ov"], dov, 0, B.n, dhv)
    lin_bwd(hc[-1], None, "hc", cache["oc"], doc, 0, B.m, dhc)
    dXv, dXc = _empty(torch, B.n, 2 * H), _empty(torch, B.m, 2 * H)
    for l in reversed(range(LAYERS)):
        # h_v[l+1] = relu([h_v[l] | a_v[l]] W_v[l] + b)
        lin_bwd(hv[l], av[l], f"v{l}", hv[l + 1], dhv, 1, B.n, dXv)
        ndhv, dav = torch.zeros((B.n, H), dtype=torch.float32, device="cuda"), _empty(torch, B.n)
        hn.check(lib.hn_gnn_split_grad(B.n, dXv.data_ptr(), ndhv.data_ptr(), dav.data_ptr(), None))
        # a_v[l] = A_c^T h_c[l+1]  ->  d h_c[l+1] += A_c d a_v[l]
        hn.check(lib.hn_gnn_spmm(B.Ac.h, 0, dav.data_ptr(), dhc.data_ptr(), 1, None))
        # h_c[l+1] = relu([h_c[l] | a_c[l]] W_c[l] + b)
        lin_bwd(hc[l], ac[l], f"c{l}", hc[l + 1], dhc, 1, B.m, dXc)
        ndhc, dac = torch.zeros((B.m, H), dtype=torch.float32, device="cuda"), _empty(torch, B.m)
        hn.check(lib.hn_gnn_split_grad(B.m, dXc.data_ptr(), ndhc.data_ptr(), dac.data_ptr(), None))
        # a_c[l] = A_r h_v[l]  ->  d h_v[l] += A_r^T d a_c[l]
        hn.check(lib.hn_gnn_spmm(B.Ar.h, 1, dac.data_ptr(), ndhv.data_ptr(), 1, None))
        dhv, dhc = ndhv, ndhc
    lin_bwd(B.Fv, None, "ev", hv[0], dhv, 1, B.n, None)
    lin_bwd(B.Fc, None, "ec", hc[0], dhc, 1, B.m, None)
    hn.check(lib.hn_gnn_check(None))
    return float(lp_v.sum().item()) / B.n + float(lp_c.sum().item()) / B.m


def train(model: Model, batches: list, epochs: int, lr: float = 1e-3, seed: int = 0, log=None):
    """Adam over the batches in a seeded order each epoch; returns the losses."""
    rng = np.random.default_rng(seed)
    losses = []
    for ep in range(epochs):
        tot = 0.0
        for i in rng.permutation(len(batches)):
            cache = forward(model, batches[i])
            tot += backward(model, batches[i], cache)
            model.adam(lr=lr)
        losses.append(tot / len(batches))
        if log:
            log(ep, losses[-1])
    return losses


def predict(model: Model, B: Batch):
    """Per LP of the batch: warm start (x, y, s) in the original space."""
    cache = forward(model, B)
    ov = cache["ov"].cpu().numpy()
    oc = cache["oc"].cpu().numpy()
    out = []
    for k in range(len(B.lps)):
        v = ov[B.n_off[k]:B.n_off[k + 1]]
        c = oc[B.m_off[k]:B.m_off[k + 1]]
        out.append((np.expm1(np.maximum(v[:, 0], 0.0)), c[:, 0].astype(np.float64),
                    np.expm1(np.maximum(v[:, 1], 0.0))))
    return out
