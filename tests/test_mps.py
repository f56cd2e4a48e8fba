"""MPS reader (hn_mps_*, host) against the reference's own MPSParser.

Each tests/golden/mps/*.mps file is read by the product reader in the
detected layout and in both forced layouts. The reader's coefficient
triplets, put through the reference's SparseMatrix::from_triplets (compiled
into oracle/_ref) or, where that library is absent, through the oracle's
restatement of it, must give the reference parser's constraint matrix bit
for bit; rows, columns, bounds, senses, ranges, types, names and the
objective sense must match exactly. The reference's results are pinned in
tests/golden/mps_reference.json (tests/golden/make_mps_golden.py) and, when
oracle/_ref is built, also recomputed live on perturbed texts.
"""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

MPS_DIR = os.path.join(ROOT, "tests", "golden", "mps")


@pytest.fixture(scope="module")
def hn():
    """The bindings without a device: the reader is host code."""
    import hnb200

    return hnb200


GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "mps_reference.json")))
CASES = sorted(GOLDEN)


def unhex(a):
    return np.array([float.fromhex(v) for v in a], dtype=np.float64)


def bits(a):
    return np.asarray(a, dtype=np.float64).view(np.uint64)


def csr_of(r, m, n):
    """Constraint matrix of the product reader's triplets, assembled with the
    reference's from_triplets semantics (the checker, not the product)."""
    if oracle.ref() is not None:
        return oracle.ref_from_triplets(m, n, r["trow"], r["tcol"], r["tval"])
    return oracle.from_triplets_port(m, n, r["trow"], r["tcol"], r["tval"])


def check_against(r, g):
    assert (r["m"], r["n"], r["maximize"]) == (g["m"], g["n"], g["maximize"])
    assert r["row_names"] == g["row_names"] and r["col_names"] == g["col_names"]
    assert r["name"] == g["name"]
    assert len(r["warnings"]) == g["warnings"]
    for k in ("c", "rhs", "lb", "ub", "range_lo", "range_hi"):
        assert np.array_equal(bits(r[k]), bits(unhex(g[k]))), k
    assert np.array_equal(r["sense"], np.array(g["sense"], dtype=np.int32))
    assert np.array_equal(r["vtype"], np.array(g["vtype"], dtype=np.int32))
    rp, ci, val = csr_of(r, r["m"], r["n"])
    assert np.array_equal(rp.astype(np.int64), np.array(g["rp"], dtype=np.int64))
    assert np.array_equal(ci.astype(np.int64), np.array(g["ci"], dtype=np.int64))
    assert np.array_equal(bits(val), bits(unhex(g["val"])))


@pytest.mark.parametrize("case", CASES)
def test_reader_matches_reference_golden(hn, case):
    name, fmt = case.rsplit(":", 1)
    text = open(os.path.join(MPS_DIR, name), "rb").read()
    check_against(hn.mps_read(text=text, fmt=int(fmt)), GOLDEN[case])


def test_reader_reads_files_and_reports_missing(hn, tmp_path):
    p = os.path.join(MPS_DIR, "free_basic.mps")
    a = hn.mps_read(path=p)
    b = hn.mps_read(text=open(p, "rb").read())
    assert a["col_names"] == b["col_names"] and np.array_equal(a["tval"], b["tval"])
    with pytest.raises(hn.HnError, match="Cannot open file"):
        hn.mps_read(path=str(tmp_path / "missing.mps"))


def test_reader_counts_records_it_reads_past(hn):
    r = hn.mps_read(text=open(os.path.join(MPS_DIR, "quad_sos.mps"), "rb").read())
    assert r["quadratic_records"] == 3 and r["sos_records"] == 2


def test_triplets_keep_file_order_and_duplicates(hn):
    text = b"ROWS\n N o\n L a\n L b\nCOLUMNS\n x a 1 b 2\n x a 3\n y b 4 a 0\nRHS\n r a 1\nENDATA\n"
    r = hn.mps_read(text=text)
    assert r["trow"].tolist() == [0, 1, 0, 1] and r["tcol"].tolist() == [0, 0, 0, 1]
    assert r["tval"].tolist() == [1.0, 2.0, 3.0, 4.0]


def _perturbed_texts():
    """Variants of the golden inputs: CRLF endings, tab separators, extra
    blank and comment lines, a trailing line without newline."""
    out = []
    for name in sorted(os.listdir(MPS_DIR)):
        if not name.endswith(".mps") or name == "lp_small.mps":
            continue
        t = open(os.path.join(MPS_DIR, name), "rb").read()
        out.append((name + ":crlf", t.replace(b"\r\n", b"\n").replace(b"\n", b"\r\n")))
        out.append((name + ":tabs", t.replace(b"  ", b"\t")))
        lines = t.split(b"\n")
        out.append((name + ":comments", b"\n".join(sum(([l, b"* note", b""] for l in lines), []))))
        out.append((name + ":nofinal", t.rstrip(b"\n")))
    return out


@pytest.mark.skipif(oracle.ref() is None, reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("fmt", [-1, 0, 1])
def test_reader_matches_live_reference_on_variants(hn, fmt):
    for label, text in _perturbed_texts():
        g = oracle.ref_mps(text, fmt)
        r = hn.mps_read(text=text, fmt=fmt)
        gj = {k: (v if not isinstance(v, np.ndarray) else v) for k, v in g.items()}
        gj = dict(gj, **{k: [float(x).hex() for x in g[k]] for k in ("c", "rhs", "lb", "ub", "range_lo",
                                                                       "range_hi", "val")})
        gj["rp"], gj["ci"] = g["rp"].tolist(), g["ci"].tolist()
        gj["sense"], gj["vtype"] = g["sense"].tolist(), g["vtype"].tolist()
        try:
            check_against(r, gj)
        except AssertionError as e:
            raise AssertionError(f"{label} fmt {fmt}: {e}") from e


def test_from_triplets_port_matches_reference():
    """The oracle's restatement of from_triplets, pinned to the reference's
    (used above when oracle/_ref is absent)."""
    if oracle.ref() is None:
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(4)
    m, n, k = 50, 70, 900
    r = rng.integers(0, m, k)
    c = rng.integers(0, n, k)
    v = rng.choice([-1.5, 0.0, 0.25, 1.0, 3.0], k)
    a = oracle.ref_from_triplets(m, n, r, c, v)
    b = oracle.from_triplets_port(m, n, r, c, v)
    for x, y in zip(a, b):
        assert np.array_equal(np.asarray(x), np.asarray(y))
