"""TEST INFRASTRUCTURE ONLY: numpy restatement of the GNN warm-start network
(the package's gnn.py, kernels hn_gnn_* of csrc/hn_gnn.cu), forward and
backward, in float64.

With bf16=True every GEMM operand is first rounded to float32 and then to
bfloat16 (round to nearest even), as the kernels stage them, so the kernels'
results differ from this restatement only by float32 accumulation order and
the rare bfloat16 rounding flips that order causes. With bf16=False it is the
exact float64 network, whose gradient tests/test_gnn.py checks against finite
differences. There is no reference counterpart (the reference has no learned
warm start), so this oracle is pinned by those finite differences only.
"""
from __future__ import annotations

import numpy as np

H = 64


def to_bf16(a) -> np.ndarray:
    """float64 -> float32 -> bfloat16 (round to nearest even), as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def csr_dense(m, n, rp, ci, val):
    A = np.zeros((m, n))
    rows = np.repeat(np.arange(m), np.diff(rp))
    np.add.at(A, (rows, np.asarray(ci, np.int64)), val)
    return A


class Net:
    """The network on one packed batch (dense A_r, A_c: test sizes only)."""

    def __init__(self, layer_shapes, params, Ar, Ac, Fv, Fc, bf16=True):
        self.shapes = layer_shapes
        self.bf16 = bf16
        self.W, self.b, off = {}, {}, 0
        for name, K in layer_shapes:
            self.W[name] = np.asarray(params[off:off + K * H], np.float64).reshape(K, H)
            self.b[name] = np.asarray(params[off + K * H:off + K * H + H], np.float64)
            off += K * H + H
        # the kernels read A's values rounded to float32
        self.Ar = np.asarray(Ar, np.float32).astype(np.float64)
        self.Ac = np.asarray(Ac, np.float32).astype(np.float64)
        self.Fv, self.Fc = np.asarray(Fv, np.float64), np.asarray(Fc, np.float64)
        self.layers = (len(layer_shapes) - 4) // 2

    def r(self, a):
        return to_bf16(a) if self.bf16 else a

    def lin(self, X, name, relu):
        Y = self.r(X) @ self.r(self.W[name]) + self.b[name]
        return np.maximum(Y, 0.0) if relu else Y

    def forward(self):
        hv = [self.lin(self.Fv, "ev", True)]
        hc = [self.lin(self.Fc, "ec", True)]
        ac, av = [], []
        for l in range(self.layers):
            ac.append(self.Ar @ hv[-1])
            hc.append(self.lin(np.hstack([hc[-1], ac[-1]]), f"c{l}", True))
            av.append(self.Ac.T @ hc[-1])
            hv.append(self.lin(np.hstack([hv[-1], av[-1]]), f"v{l}", True))
        self.cache = dict(hv=hv, hc=hc, ac=ac, av=av, ov=self.lin(hv[-1], "hv", False),
                          oc=self.lin(hc[-1], "hc", False))
        return self.cache

    def loss(self, Tv, Tc):
        c = self.cache
        ev = c["ov"][:, :2] - Tv
        ec = c["oc"][:, :1] - Tc[:, :1]
        return float((ev ** 2).sum() / Tv.shape[0] + (ec ** 2).sum() / Tc.shape[0])

    def backward(self, Tv, Tc):
        c = self.cache
        n, m = Tv.shape[0], Tc.shape[0]
        grads = {}

        def lin_bwd(X, name, Y, dY, relu, want_dx=True):
            G = dY * (Y > 0) if relu else dY
            grads[name] = (self.r(X).T @ self.r(G), G.sum(0))
            return self.r(G) @ self.r(self.W[name]).T if want_dx else None

        dov = np.zeros_like(c["ov"])
        dov[:, :2] = 2.0 * (c["ov"][:, :2] - Tv) / n
        doc = np.zeros_like(c["oc"])
        doc[:, :1] = 2.0 * (c["oc"][:, :1] - Tc[:, :1]) / m
        hv, hc, ac, av = c["hv"], c["hc"], c["ac"], c["av"]
        dhv = lin_bwd(hv[-1], "hv", c["ov"], dov, False)
        dhc = lin_bwd(hc[-1], "hc", c["oc"], doc, False)
        for l in reversed(range(self.layers)):
            dX = lin_bwd(np.hstack([hv[l], av[l]]), f"v{l}", hv[l + 1], dhv, True)
            ndhv, dav = dX[:, :H].copy(), dX[:, H:]
            dhc = dhc + self.Ac @ dav
            dX = lin_bwd(np.hstack([hc[l], ac[l]]), f"c{l}", hc[l + 1], dhc, True)
            ndhc, dac = dX[:, :H].copy(), dX[:, H:]
            ndhv = ndhv + self.Ar.T @ dac
            dhv, dhc = ndhv, ndhc
        lin_bwd(self.Fv, "ev", hv[0], dhv, True, False)
        lin_bwd(self.Fc, "ec", hc[0], dhc, True, False)
        flat = []
        for name, K in self.shapes:
            gw, gb = grads[name]
            flat += [gw.reshape(-1), gb]
        return np.concatenate(flat)
