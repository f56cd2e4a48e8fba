"""Crossover from the GPU IPM's endpoint.

hn_lp_solve (the GPU barrier) -> hn_crossover_basis -> the reference's
simplex polish (SimplexSolver::solve_with_basis, then a cold solve if the
warm start gives no verdict) must reach the verdict and vertex objective of
the reference's own InteriorPointSolver with crossover on.
"""
import numpy as np
import pytest

import lpgen
import oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(oracle.ref() is None, reason="oracle/_ref not built (reference sources absent)")]


@pytest.mark.parametrize("m,n,seed,bounded", [(40, 100, 1, False), (60, 150, 2, True), (120, 300, 4, True)])
def test_gpu_barrier_endpoint_polishes_to_reference_crossover(hn, m, n, seed, bounded):
    lp = lpgen.lp_uniform(m, n, 5, seed=seed)
    lb = np.zeros(n)
    ub = np.full(n, np.inf)
    if bounded:
        ub[::3] = 1.0 + (np.arange(0, n, 3) % 4)
    gpu = hn.lp_solve(lp, lb=lb, ub=ub)
    assert gpu["status_name"] == "OPTIMAL"
    vs = hn.crossover_basis(gpu["x"], lb, ub)
    ours = oracle.ref_crossover_polish(lp, vs, gpu["status"], lb=lb, ub=ub)
    ref = oracle.ref_ipm_solve(lp, lb=lb, ub=ub, crossover=True)
    assert ours["status"] == ref["status"] == 1
    assert abs(ours["objective"] - ref["objective"]) <= 1e-9 * (1.0 + abs(ref["objective"]))
