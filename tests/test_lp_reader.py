"""LP-format reader (hn_lp_read_*, host) against the reference's LPParser.

Each tests/golden/lp/*.lp file is read by the product reader. Where the
reference reads it, the columns (in the reference's creation order), rows,
bounds, types, senses and the constraint matrix (the reader's triplets put
through from_triplets: the reference's when oracle/_ref is built, else the
oracle's restatement) must match bit for bit; where the reference reports
errors, the product read must fail. Pinned in tests/golden/lp_reference.json
(tests/golden/make_mps_golden.py) and, when oracle/_ref is built, recomputed
live on perturbed texts.
"""
import json
import os

import numpy as np
import pytest

import oracle
from test_mps import check_against

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LP_DIR = os.path.join(ROOT, "tests", "golden", "lp")
GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "lp_reference.json")))


@pytest.fixture(scope="module")
def hn():
    """The bindings without a device: the reader is host code."""
    import hnb200

    return hnb200


def _check(hn, text, g, label):
    if not g["success"]:
        with pytest.raises(hn.HnError, match="LP text rejected"):
            hn.lp_read(text=text)
        return
    try:
        check_against(hn.lp_read(text=text), g)
    except AssertionError as e:
        raise AssertionError(f"{label}: {e}") from e


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_lp_reader_matches_reference_golden(hn, name):
    _check(hn, open(os.path.join(LP_DIR, name), "rb").read(), GOLDEN[name], name)


def test_lp_reader_reads_files(hn, tmp_path):
    p = os.path.join(LP_DIR, "basic.lp")
    a = hn.lp_read(path=p)
    assert a["col_names"] == ["x", "y", "z", "w"] and a["maximize"] == 1
    with pytest.raises(hn.HnError, match="Cannot open file"):
        hn.lp_read(path=str(tmp_path / "missing.lp"))


def _variants():
    out = []
    for name in sorted(os.listdir(LP_DIR)):
        if not name.endswith(".lp") or name == "lp_small.lp":
            continue
        t = open(os.path.join(LP_DIR, name), "rb").read()
        out.append((name + ":crlf", t.replace(b"\r\n", b"\n").replace(b"\n", b"\r\n")))
        out.append((name + ":tabs", t.replace(b" ", b"\t")))
        lines = t.split(b"\n")
        out.append((name + ":comments", b"\n".join(sum(([l, b"\\ note", b"** more", b""] for l in lines), []))))
        out.append((name + ":nofinal", t.rstrip(b"\n")))
        out.append((name + ":spaced", t.replace(b"<=", b" <= ").replace(b">=", b" >= ").replace(b":", b" : ")))
    return out


def _as_golden(g):
    out = dict(g)
    for k in ("c", "rhs", "lb", "ub", "range_lo", "range_hi", "val"):
        out[k] = [float(x).hex() for x in g[k]]
    for k in ("rp", "ci", "sense", "vtype"):
        out[k] = np.asarray(g[k]).tolist()
    return out


@pytest.mark.skipif(oracle.ref() is None, reason="oracle/_ref not built (reference sources absent)")
def test_lp_reader_matches_live_reference_on_variants(hn):
    for label, text in _variants():
        _check(hn, text, _as_golden(oracle.ref_mps(text, lp_format=True)), label)
