"""GPU: the relative KKT residual of every solve and the tightening past the
reference's stopping rule.

The reference stops on absolute tests of its scaled standard form
(core/lp/interior_point.cpp:525-530), which can leave a relative duality gap
above 1e-8. Every plain and batched solve here measures, on the device, the
relative KKT residual of the unscaled LP (hn_ipm_kkt):

    max(||Ax-b||/(1+||b||), ||A^T y + s - c||/(1+||c||), |c^T x - b^T y|/(1+|c^T x|))

and keeps iterating past the reference's stop until it is <= 1e-8 (or 10 more
iterations ran, returning the better iterate). Checked here:
  * every solve of a mixed batch whose reference test held, and the plain
    solves, end OPTIMAL at <= 1e-8;
  * the device measure agrees with a numpy restatement on the original LP
    (primal part and gap from x and the dual estimate y; dual feasibility of
    s = c - A^T y bounded by the dual part);
  * the trajectory up to the reference's stop is unchanged: the iteration at
    which the reference's rule first holds equals the iteration count of the
    same batch solved with the reference's rule alone, and the objectives agree
    within 1e-8;
  * with an unreachable tolerance the extra iterations are bounded and the
    result stays the reference rule's.
"""
import json
import os

import numpy as np
import pytest

import lpgen

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def rel(a, b):
    return abs(a - b) / (1.0 + abs(b))


def numpy_kkt_parts(lp, x, y):
    """Primal part, gap part and dual infeasibility of s = c - A^T y for an
    LP min c^T x, A x = b, x >= 0 (numpy, float64)."""
    m, n = lp["m"], lp["n"]
    rows = np.repeat(np.arange(m), np.diff(lp["rp"]))
    ax = np.zeros(m)
    np.add.at(ax, rows, lp["val"] * x[lp["ci"]])
    aty = np.zeros(n)
    np.add.at(aty, lp["ci"], lp["val"] * y[rows])
    b, c = lp["b"], lp["c"]
    primal = np.max(np.abs(ax - b)) / (1.0 + np.max(np.abs(b)))
    cx = float(c @ x)
    gap = abs(cx - float(b @ y)) / (1.0 + abs(cx))
    s = c - aty
    dual_infeas = max(0.0, float(np.max(-s))) / (1.0 + np.max(np.abs(c)))
    return primal, gap, dual_infeas


def check_measure(lp, x, y, kkt, parts):
    p_np, g_np, dinf = numpy_kkt_parts(lp, x, y)
    p_dev, d_dev, g_dev = parts
    assert kkt == max(p_dev, d_dev, g_dev)
    assert abs(p_np - p_dev) <= 1e-12, (p_np, p_dev)
    assert abs(g_np - g_dev) <= 1e-11, (g_np, g_dev)
    # s = z - rd in the original scaling, z > 0: -s <= |rd|
    assert dinf <= d_dev * (1 + 1e-6) + 1e-15, (dinf, d_dev)


@pytest.mark.parametrize("args", [(60, 150, 8, 3), (200, 500, 8, 4), (500, 1250, 6, 11)])
def test_plain_solve_reaches_relative_kkt(hn, args):
    lp = lpgen.lp_uniform(*args)
    r = hn.lp_solve(lp)
    assert r["status_name"] == "OPTIMAL", r
    assert r["kkt"] <= 1e-8, (r["kkt"], r["kkt_parts"])
    assert 0 <= r["reference_iterations"] <= r["iterations"] <= r["reference_iterations"] + 10
    check_measure(lp, r["x"], r["y"], r["kkt"], r["kkt_parts"])
    ref_rule = hn.lp_solve(lp, kkt_tol=0.0)
    assert ref_rule["iterations"] == r["reference_iterations"]
    assert rel(r["objective"], ref_rule["objective"]) <= 1e-8


def test_plain_m2000_lp_at_relative_kkt_with_the_reference_objective(hn):
    path = os.path.join(HERE, "golden", "reference_ipm_c0.json")
    if not os.path.exists(path):
        pytest.skip("reference result for the m=2000 LP not generated")
    ref = json.load(open(path))["lp_uniform_2000_5000_8_seed0"]
    r = hn.lp_solve(lpgen.lp_uniform(2000, 5000, 8, 0))
    assert r["status"] == ref["status"] == 1
    assert r["kkt"] <= 1e-8, (r["kkt"], r["kkt_parts"])
    assert rel(r["objective"], ref["objective"]) <= 1e-8, (r["objective"], ref["objective"])


def mixed_batch(k=20, seed=21):
    sizes = lpgen.batch_sizes(k, 30, 400, seed=seed)
    return [lpgen.lp_uniform(int(mm), int(round(2.5 * mm)), 6, 500 + i) for i, mm in enumerate(sizes)]


def test_batch_every_solve_reaches_relative_kkt(hn):
    """Every instance whose reference test held reaches <= 1e-8; an instance
    the reference accepts only by its relaxed test at the iteration limit
    (interior_point.cpp:727-753) keeps the reference algorithm's point."""
    lps = mixed_batch()
    r = hn.lp_solve_batch(lps)
    base = hn.lp_solve_batch(lps, kkt_tol=0.0)
    strict = 0
    for k, lp in enumerate(lps):
        assert r["status"][k] == 1 and base["status"][k] == 1, k
        if r["reference_iterations"][k] >= 0:
            strict += 1
            assert r["kkt"][k, 0] <= 1e-8, (k, r["kkt"][k])
            # the same trajectory up to the reference's stop
            assert r["reference_iterations"][k] == base["iterations"][k], k
            assert r["reference_iterations"][k] <= r["iterations"][k] <= r["reference_iterations"][k] + 10
        else:
            assert r["iterations"][k] == base["iterations"][k] == 100, k
            assert np.array_equal(r["kkt"][k], base["kkt"][k]), k
        assert rel(r["objective"][k], base["objective"][k]) <= 1e-8, k
        c0, c1 = r["col_off"][k], r["col_off"][k + 1]
        r0, r1 = r["row_off"][k], r["row_off"][k + 1]
        check_measure(lp, r["x"][c0:c1], r["y"][r0:r1], r["kkt"][k, 0], r["kkt"][k, 1:])
    assert strict >= len(lps) - 2
    # the reference's rule alone still measures the residual
    assert np.all(np.isfinite(base["kkt"][:, 0]))


def test_batch_matches_plain_kkt(hn):
    lps = mixed_batch(6, seed=4)
    r = hn.lp_solve_batch(lps)
    for k, lp in enumerate(lps):
        p = hn.lp_solve(lp)
        # the plain IPM factorises on the host, the batch on the GPU: same
        # status and objective, not necessarily the same iteration count
        assert p["status"] == r["status"][k] == 1, k
        assert rel(p["objective"], r["objective"][k]) <= 1e-8, k
        assert p["kkt"] <= 1e-8 and r["kkt"][k, 0] <= 1e-8


def test_unreachable_tolerance_bounds_the_extra_iterations(hn):
    lps = mixed_batch(8, seed=9)
    base = hn.lp_solve_batch(lps, kkt_tol=0.0)
    r = hn.lp_solve_batch(lps, kkt_tol=1e-300, kkt_extra=3)
    for k in range(len(lps)):
        assert r["status"][k] == base["status"][k] == 1
        assert r["reference_iterations"][k] == base["iterations"][k]
        assert r["iterations"][k] <= base["iterations"][k] + 3
        # never worse than what the reference's rule accepted
        assert r["kkt"][k, 0] <= base["kkt"][k, 0]
        assert rel(r["objective"][k], base["objective"][k]) <= 1e-8
    p = hn.lp_solve(lps[0], kkt_tol=1e-300, kkt_extra=3)
    assert p["status_name"] == "OPTIMAL" and p["iterations"] <= p["reference_iterations"] + 3
