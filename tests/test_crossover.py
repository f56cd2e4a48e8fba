"""Crossover seam (hn_crossover_basis, host) against the reference.

The reference's InteriorPointSolver with crossover hands SimplexSolver::
solve_with_basis a warm basis built from the barrier endpoint
(interior_point.cpp:825-842). hn_crossover_basis computes that basis; here
it is pinned (a) element for element against a restatement of the rule,
infinite bounds included, and (b) end to end: the reference barrier's
endpoint (crossover off) -> hn_crossover_basis -> the reference's polish
gives the status and objective of the reference solver with crossover on.
"""
import numpy as np
import pytest

import lpgen
import oracle


@pytest.fixture(scope="module")
def hn():
    """The bindings without a device: the rule is host code."""
    import hnb200

    return hnb200


def _rule(x, lb, ub):
    """The reference's rule, restated: tolerance 1e-6 (1 + max(|lb|, |ub|)),
    lower bound tested first (an infinite bound makes it infinite)."""
    out = np.zeros(x.shape[0], dtype=np.int32)
    with np.errstate(invalid="ignore"):
        tol = 1e-6 * (1.0 + np.maximum(np.abs(lb), np.abs(ub)))
        at_lo = x <= lb + tol
        at_hi = x >= ub - tol
    out[at_hi] = 1
    out[at_lo] = -1
    return out


def test_basis_rule_matches_restatement(hn):
    rng = np.random.default_rng(11)
    n = 5000
    lb = rng.choice([0.0, -1.0, -np.inf, 2.5], n)
    ub = np.where(rng.random(n) < 0.5, np.inf, lb + rng.choice([0.0, 1e-7, 1.0, 10.0], n))
    # points on, near and away from the bounds
    x = np.where(rng.random(n) < 0.3, lb, np.where(rng.random(n) < 0.5, ub, rng.normal(1.0, 2.0, n)))
    x = np.where(np.isfinite(x), x, 0.0) + rng.choice([0.0, 5e-7, -5e-7, 3e-6], n)
    got = hn.crossover_basis(x, lb, ub)
    assert np.array_equal(got, _rule(x, lb, ub))
    # a finite lower bound with no upper bound: always offered at the lower bound
    assert hn.crossover_basis([5.0], [0.0], [np.inf]).tolist() == [-1]
    assert hn.crossover_basis([0.5], [0.0], [1.0]).tolist() == [0]
    assert hn.crossover_basis([1.0], [0.0], [1.0]).tolist() == [1]


@pytest.mark.skipif(oracle.ref() is None, reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("m,n,seed,bounded", [(40, 100, 1, False), (60, 150, 2, True), (30, 90, 3, True)])
def test_polish_from_barrier_endpoint_matches_reference_crossover(hn, m, n, seed, bounded):
    lp = lpgen.lp_uniform(m, n, 5, seed=seed)
    lb = np.zeros(n)
    ub = np.full(n, np.inf)
    if bounded:
        ub[::3] = 1.0 + (np.arange(0, n, 3) % 4)  # some upper bounds, some of them active
    barrier = oracle.ref_ipm_solve(lp, lb=lb, ub=ub, crossover=False)
    vs = hn.crossover_basis(barrier["x"], lb, ub)
    ours = oracle.ref_crossover_polish(lp, vs, barrier["status"], lb=lb, ub=ub)
    ref = oracle.ref_ipm_solve(lp, lb=lb, ub=ub, crossover=True)
    assert ours["status"] == ref["status"]
    assert abs(ours["objective"] - ref["objective"]) <= 1e-9 * (1.0 + abs(ref["objective"]))
