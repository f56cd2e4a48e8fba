"""Device CSR from MPS triplets (hn_csr_create_coo) against the reference.

The reference's MPSParser builds its constraint matrix with
SparseMatrix::from_triplets; the product reads the same file with hn_mps_*
and sorts the triplets into CSR on the device. Bit-exact against the
reference parser's matrices pinned in tests/golden/mps_reference.json, and
against the oracle's from_triplets restatement on seeded random triplets
(unsorted, repeated keys, cancelling pairs, empty rows and columns).
"""
import json
import os

import numpy as np
import pytest

import lpgen
import oracle

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MPS_DIR = os.path.join(ROOT, "tests", "golden", "mps")
GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "mps_reference.json")))


def bits(a):
    return np.asarray(a, dtype=np.float64).view(np.uint64)


@pytest.mark.parametrize("case", sorted(k for k in GOLDEN if k.endswith(":-1")))
def test_read_mps_device_csr_matches_reference_parser(hn, case):
    name = case.rsplit(":", 1)[0]
    g = GOLDEN[case]
    lp = hn.read_mps(path=os.path.join(MPS_DIR, name))
    assert (lp["m"], lp["n"]) == (g["m"], g["n"])
    assert np.array_equal(lp["rp"].astype(np.int64), np.array(g["rp"], dtype=np.int64))
    assert np.array_equal(lp["ci"].astype(np.int64), np.array(g["ci"], dtype=np.int64))
    assert np.array_equal(bits(lp["val"]), bits([float.fromhex(v) for v in g["val"]]))


@pytest.mark.parametrize("m,n,count,seed", [(1, 1, 0, 0), (5, 1, 40, 1), (1, 9, 40, 2), (300, 200, 5000, 3),
                                            (20000, 3000, 300000, 4), (4096, 70000, 250000, 5)])
def test_coo_to_csr_matches_from_triplets(hn, m, n, count, seed):
    rng = np.random.default_rng(seed)
    r = rng.integers(0, m, count)
    c = rng.integers(0, n, count)
    v = rng.standard_normal(count)
    if count:
        # repeated keys in scattered positions, some cancelling exactly
        k = max(count // 10, 1)
        src = rng.integers(0, count, k)
        dst = rng.integers(0, count, k)
        r[dst], c[dst] = r[src], c[src]
        v[dst[: k // 2]] = -v[src[: k // 2]]
        v[rng.integers(0, count, k // 4)] = 0.0
    A = hn.Csr.from_coo(m, n, r, c, v)
    rp, ci, val = A.export()
    erp, eci, evl = oracle.from_triplets_port(m, n, r, c, v)
    assert np.array_equal(rp, erp) and np.array_equal(ci, eci)
    assert np.array_equal(bits(val), bits(evl))
    # the device A^T of the triplet-built matrix equals the one hn_csr_create builds
    B = hn.Csr(m, n, erp, eci, evl)
    for x, y in zip(A.export(trans=1), B.export(trans=1)):
        assert np.array_equal(np.asarray(x).view(np.uint64), np.asarray(y).view(np.uint64))
    A.close()
    B.close()


def test_coo_rejects_out_of_range_triplets(hn):
    with pytest.raises(hn.HnError, match="outside"):
        hn.Csr.from_coo(3, 3, [0, 3], [0, 0], [1.0, 2.0])
    with pytest.raises(hn.HnError, match="outside"):
        hn.Csr.from_coo(3, 3, [0, 1], [0, -1], [1.0, 2.0])


def test_mps_file_solves_like_the_generated_lp(hn):
    """lp_small.mps (written from a seeded generator LP, some coefficients
    split in two entries, some cancelling pairs) read through hn_mps and the
    device CSR, solved by the GPU IPM: same status, objective within the
    IPM tolerance of the generator's own LP."""
    lp_mps = hn.read_mps(path=os.path.join(MPS_DIR, "lp_small.mps"))
    base = lpgen.lp_uniform(120, 300, 6, seed=77)
    r1 = hn.lp_solve(lp_mps, sense=lp_mps["sense"], lb=lp_mps["lb"], ub=lp_mps["ub"],
                     maximize=lp_mps["maximize"])
    ub = np.full(300, np.inf)
    ub[::5] = 10.0 + np.arange(0, 300, 5) % 7
    r0 = hn.lp_solve(base, ub=ub)
    assert r1["status_name"] == r0["status_name"] == "OPTIMAL"
    assert abs(r1["objective"] - r0["objective"]) <= 1e-8 * (1.0 + abs(r0["objective"]))
