"""GPU: the IPM warm start (no reference counterpart: the reference's IPM
always starts from Mehrotra's default point, interior_point.cpp:443-453).

A warm start is mapped to the scaled standard form, shifted to strict
interiority and taken only when its relative KKT residual is below the
default start's; whatever start is taken, the solve must end with the
reference's status and objective (1e-8 relative)."""
import numpy as np
import pytest

import lpgen

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs(a - b) / (1.0 + abs(b))


def test_warm_from_solution_is_taken_and_saves_iterations(hn):
    lp = lpgen.lp_uniform(200, 500, 8, 4)
    cold = hn.lp_solve(lp)
    assert cold["status"] == 1 and not cold["warm_start_used"]
    # the barrier's dual estimate: A^T y + s = c, s ~ 0 where x > 0
    A_T_y = lpgen.csr_tmatvec(lp["rp"], lp["ci"], lp["val"], cold["y"], lp["n"])
    assert np.max(np.abs(A_T_y + cold["s"] - lp["c"])) <= 1e-9 * (1 + np.max(np.abs(lp["c"])))
    assert abs(cold["x"] @ cold["s"]) <= 1e-6 * (1 + abs(cold["objective"]))
    warm = hn.lp_solve(lp, x0=cold["x"], y0=cold["y"], s0=cold["s"])
    assert warm["warm_start_used"] and warm["kkt_warm"] < warm["kkt_default"]
    assert warm["status"] == 1 and rel(warm["objective"], cold["objective"]) <= 1e-8
    assert warm["iterations"] < cold["iterations"]


def test_interior_feasible_point_is_taken(hn):
    lp = lpgen.lp_uniform(300, 750, 8, 12)
    cold = hn.lp_solve(lp)
    warm = hn.lp_solve(lp, x0=lp["x0"], y0=lp["y0"])  # s from c - A^T y
    assert warm["warm_start_used"]
    assert warm["status"] == cold["status"] == 1 and rel(warm["objective"], cold["objective"]) <= 1e-8


def test_bad_warm_start_falls_back_to_default(hn):
    lp = lpgen.lp_uniform(200, 500, 8, 4)
    cold = hn.lp_solve(lp)
    bad = hn.lp_solve(lp, x0=np.full(lp["n"], 1e9), y0=np.full(lp["m"], -1e9))
    assert not bad["warm_start_used"] and bad["kkt_warm"] >= bad["kkt_default"]
    assert bad["iterations"] == cold["iterations"] and bad["objective"] == cold["objective"]
    wrong = hn.lp_solve(lp, x0=np.ones(3))  # wrong size: ignored
    assert not wrong["warm_start_used"] and wrong["objective"] == cold["objective"]


def test_batch_warm_matches_plain_warm(hn):
    lps = [lpgen.lp_uniform(int(m), int(2.5 * m), 6, 300 + i) for i, m in enumerate((60, 140, 250))]
    x0s = [lp["x0"] for lp in lps]
    y0s = [lp["y0"] for lp in lps]
    s0s = [lp["s0"] for lp in lps]
    r = hn.lp_solve_batch(lps, x0s=x0s, y0s=y0s, s0s=s0s)
    for k, lp in enumerate(lps):
        p = hn.lp_solve(lp, x0=x0s[k], y0=y0s[k], s0=s0s[k])
        assert r["warm_used"][k] == p["warm_start_used"]
        assert r["status"][k] == p["status"] == 1 and rel(r["objective"][k], p["objective"]) <= 1e-8


def test_branch_and_bound_node_batch_warm_from_the_parent(hn):
    """Branch-and-bound style nodes of one base LP (each tightens 1-8
    variable bounds: ub = floor or lb = ceil of a perturbed x0_j, so the
    standard forms gain upper-bound rows of their own and differ in shape),
    solved in one batch warm-started from the parent's barrier solution
    (x and the dual estimate y): every node ends with the status and
    objective of its own cold plain solve (1e-8), at relative KKT <= 1e-8,
    and the parent's point is taken as the start for most nodes."""
    base = lpgen.lp_uniform(300, 720, 8, 31)
    parent = hn.lp_solve(base)
    assert parent["status"] == 1
    nodes = lpgen.bb_nodes(base, 12, kmax=8, seed=77)
    lbs, ubs = [lb for lb, _ in nodes], [ub for _, ub in nodes]
    r = hn.lp_solve_batch([base] * len(nodes), lbs=lbs, ubs=ubs, x0s=[parent["x"]] * len(nodes),
                          y0s=[parent["y"]] * len(nodes))
    assert int(r["warm_used"].sum()) >= len(nodes) // 2
    for k, (lb, ub) in enumerate(nodes):
        cold = hn.lp_solve(base, lb=lb, ub=ub)
        assert r["status"][k] == cold["status"], (k, r["status"][k], cold["status"])
        if cold["status"] == 1:
            assert rel(r["objective"][k], cold["objective"]) <= 1e-8, (k, r["objective"][k], cold["objective"])
            assert r["kkt"][k, 0] <= 1e-8, (k, r["kkt"][k])
            # a tightened bound can only raise the minimum
            assert r["objective"][k] >= parent["objective"] - 1e-8 * (1 + abs(parent["objective"]))
