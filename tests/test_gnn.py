"""CPU: the GNN oracle's backward (oracle/gnn_oracle.py, exact float64 mode)
against central finite differences of its loss, and the package's host-side
data preparation (features, targets, packing)."""
import numpy as np

import gnn
import gnn_oracle as GO
import lpgen


def small_net(bf16=False, seed=0):
    lps = [lpgen.lp_uniform(12, 30, 3, 5), lpgen.lp_uniform(9, 20, 3, 6)]
    rp, ci, m_off, n_off = gnn.pack(lps)
    vr, vc = zip(*(gnn.normalised_values(lp) for lp in lps))
    m, n = int(m_off[-1]), int(n_off[-1])
    Ar = GO.csr_dense(m, n, rp, ci, np.concatenate(vr))
    Ac = GO.csr_dense(m, n, rp, ci, np.concatenate(vc))
    F = [gnn.features(lp) for lp in lps]
    rng = np.random.default_rng(seed)
    sols = [(rng.uniform(0, 2, lp["n"]), rng.standard_normal(lp["m"]), rng.uniform(0, 1, lp["n"])) for lp in lps]
    T = [gnn.targets(*s) for s in sols]
    Tv = np.concatenate([t[0] for t in T]).astype(np.float64)
    Tc = np.concatenate([t[1] for t in T]).astype(np.float64)
    params = gnn.init_params(seed).astype(np.float64)
    net = GO.Net(gnn.layer_shapes(), params, Ar, Ac, np.concatenate([f[0] for f in F]),
                 np.concatenate([f[1] for f in F]), bf16=bf16)
    return net, params, Tv, Tc, Ar, Ac


def test_oracle_gradient_matches_finite_differences():
    net, params, Tv, Tc, Ar, Ac = small_net()
    net.forward()
    g = net.backward(Tv, Tc)
    rng = np.random.default_rng(1)
    offs, size = gnn.param_offsets()
    assert g.size == size == params.size
    # a few weights and biases of every layer
    idx = []
    for name, (o, K) in offs.items():
        idx += list(rng.integers(o, o + K * 64, 3)) + [o + K * 64 + int(rng.integers(0, 64))]
    eps = 1e-6
    for i in idx:
        p1, p2 = params.copy(), params.copy()
        p1[i] += eps
        p2[i] -= eps
        l1 = GO.Net(gnn.layer_shapes(), p1, Ar, Ac, net.Fv, net.Fc, bf16=False)
        l1.forward()
        l2 = GO.Net(gnn.layer_shapes(), p2, Ar, Ac, net.Fv, net.Fc, bf16=False)
        l2.forward()
        fd = (l1.loss(Tv, Tc) - l2.loss(Tv, Tc)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 1e-40, 3.0e38])
    r = GO.to_bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2.0 ** -6 and r[3] == -2.5
    assert np.all(np.abs(r - x) <= np.abs(x) * 2.0 ** -8 + 1e-38)


def test_features_targets_and_packing():
    lps = [lpgen.lp_uniform(10, 25, 3, 1), lpgen.lp_uniform(7, 18, 3, 2)]
    rp, ci, m_off, n_off = gnn.pack(lps)
    assert list(m_off) == [0, 10, 17] and list(n_off) == [0, 25, 43]
    assert rp[0] == 0 and rp[-1] == len(ci) == len(lps[0]["ci"]) + len(lps[1]["ci"])
    assert ci[len(lps[0]["ci"]):].min() >= 25
    Fv, Fc = gnn.features(lps[0])
    assert Fv.shape == (25, gnn.FEAT) and Fc.shape == (10, gnn.FEAT) and np.all(Fv[:, 4] == 1)
    Tv, Tc = gnn.targets(np.array([0.0, 1.0]), np.array([-1.0]), np.array([2.0, -1.0]))
    assert np.allclose(Tv, [[0, np.log1p(2.0)], [np.log1p(1.0), 0]]) and np.allclose(Tc, [[-1, 0]])
