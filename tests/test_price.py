"""CPU: the pricing restatement (oracle/hn_oracle.c) against the reference's own
SimplexSolver pricing members (core/lp/simplex.cpp:25-35, 1225-1361), driven
through oracle/ref_simplex_shim.cpp."""
import numpy as np
import pytest

import lpgen
import oracle as O

pytestmark = pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built")


def pricing_state(m=120, n=300, seed=7, ties=False):
    lp = lpgen.lp_uniform(m, n, 6, seed)
    rng = np.random.default_rng(seed)
    y = rng.standard_normal(m)
    cost = rng.standard_normal(n)
    nonbasis = np.arange(n, dtype=np.int32)
    nonbasis[rng.choice(n, size=m // 2, replace=False)] = -1
    artificial = (rng.random(n) < 0.1).astype(np.uint8)
    w = rng.uniform(0.5, 3.0, n)
    w[rng.choice(n, 8, replace=False)] = [0.0, -1.0, np.inf, np.nan, 1e-300, 0.0, 2.0, 4.0]
    if ties:
        cost = np.round(cost * 2) / 2
        w[:] = 1.0
    return lp, y, cost, nonbasis, artificial, w


def test_reduced_costs_port_matches_reference():
    lp, y, cost, *_ = pricing_state()
    a = O.price_reduced_costs(lp["m"], lp["n"], lp["rp"], lp["ci"], lp["val"], y, cost)
    b = O.ref_price_reduced_costs(lp["m"], lp["n"], lp["rp"], lp["ci"], lp["val"], y, cost)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("zero_rows", [False, True])
def test_devex_update_port_matches_reference(zero_rows):
    lp, y, cost, nonbasis, artificial, w = pricing_state(seed=11)
    w = np.abs(np.nan_to_num(w, nan=1.0, posinf=1.0))
    u = np.random.default_rng(3).standard_normal(lp["m"])
    if zero_rows:
        u[::3] = 0.0
    a, _ = O.price_devex_update(lp["m"], lp["n"], lp["rp"], lp["ci"], lp["val"], u, nonbasis, w)
    b = O.ref_price_devex_update(lp["m"], lp["n"], lp["rp"], lp["ci"], lp["val"], u, nonbasis, w)
    assert np.array_equal(a, b)
    # u = 0: s = 0 and the weights stay as they were
    a0, _ = O.price_devex_update(lp["m"], lp["n"], lp["rp"], lp["ci"], lp["val"], np.zeros(lp["m"]), nonbasis, w)
    assert np.array_equal(a0, w)


@pytest.mark.parametrize("ties", [False, True])
@pytest.mark.parametrize("phase1,maximize", [(False, False), (True, False), (False, True)])
def test_ranked_and_bland_port_match_reference(ties, phase1, maximize):
    lp, y, cost, nonbasis, artificial, w = pricing_state(seed=5, ties=ties)
    rc = O.price_reduced_costs(lp["m"], lp["n"], lp["rp"], lp["ci"], lp["val"], y, cost)
    if ties:
        rc = np.round(rc * 4) / 4
    cnt, order = O.price_ranked(rc, w, nonbasis, artificial, phase1, maximize)
    rcnt, rorder = O.ref_price_ranked(rc, w, nonbasis, artificial, phase1, maximize)
    assert cnt == rcnt and cnt > 0
    assert np.array_equal(order[:cnt], rorder)
    assert O.ref_price_select(rc, w, nonbasis, artificial, phase1, maximize, rule=1) == order[0]
    bl = O.price_bland(rc, nonbasis, artificial, phase1, maximize)
    assert O.ref_price_select(rc, w, nonbasis, artificial, phase1, maximize, rule=0) == bl


def test_no_improving_column():
    n = 50
    rc = np.abs(np.random.default_rng(1).standard_normal(n))
    nb = np.arange(n, dtype=np.int32)
    art = np.zeros(n, dtype=np.uint8)
    cnt, order = O.price_ranked(rc, np.ones(n), nb, art)
    assert cnt == 0 and order[0] == -1
    assert O.ref_price_select(rc, np.ones(n), nb, art, rule=1) == -1
    assert O.price_bland(rc, nb, art) == -1 == O.ref_price_select(rc, np.ones(n), nb, art, rule=0)


def test_extract_column_port_matches_reference_edge_weight():
    lp = lpgen.lp_uniform(80, 200, 6, 9)
    for j in (0, 17, 199):
        col = O.extract_column(lp["m"], lp["rp"], lp["ci"], lp["val"], j)
        n2 = 1.0
        for v in col:
            n2 += v * v
        assert n2 == O.ref_price_edge_weight(lp["m"], lp["n"], lp["rp"], lp["ci"], lp["val"], j)
        assert np.count_nonzero(col) == 6
