"""Writes tests/golden/mps_reference.json: the reference's own MPS reader
(model::MPSParser::parse_string, compiled into oracle/_ref) run on every
tests/golden/mps/*.mps file, in the layout it detects and in both forced
layouts. Doubles are stored as float.hex strings (bit-exact). Also writes
the generated instance lp_small.mps (a seeded LP of the C0 generator, free
layout, with repeated and cancelling coefficients) before reading it.

Run from the repository root after `make -C oracle ref`:
    python tests/golden/make_mps_golden.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "indigenous-cpu-gpu-optimization-engine-for-indian-industry_b200"))
import lpgen  # noqa: E402
import oracle  # noqa: E402

MPS_DIR = os.path.join(ROOT, "tests", "golden", "mps")
OUT = os.path.join(ROOT, "tests", "golden", "mps_reference.json")


def write_lp_small(path):
    lp = lpgen.lp_uniform(120, 300, 6, seed=77)
    rng = np.random.default_rng(78)
    lines = ["NAME LPSMALL", "ROWS", " N obj"] + [f" E r{i}" for i in range(lp["m"])] + ["COLUMNS"]
    rp, ci, val = lp["rp"], lp["ci"], lp["val"]
    cols = [[] for _ in range(lp["n"])]
    for i in range(lp["m"]):
        for k in range(int(rp[i]), int(rp[i + 1])):
            cols[int(ci[k])].append((i, float(val[k])))
    for j in range(lp["n"]):
        lines.append(f"    v{j} obj {float(lp['c'][j])!r}")
        for i, a in cols[j]:
            if rng.random() < 0.1:  # split the coefficient in two entries
                h = float(np.float64(a) * 0.375)
                lines.append(f"    v{j} r{i} {h!r} r{i} {a - h!r}")
            else:
                lines.append(f"    v{j} r{i} {a!r}")
        if rng.random() < 0.05:  # a cancelling pair
            i = int(rng.integers(lp["m"]))
            lines.append(f"    v{j} r{i} 0.25 r{i} -0.25")
    lines.append("RHS")
    lines += [f"    rhs r{i} {float(lp['b'][i])!r}" for i in range(lp["m"])]
    lines += ["BOUNDS"] + [f" UP bnd v{j} {10.0 + j % 7}" for j in range(0, lp["n"], 5)] + ["ENDATA"]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def hx(a):
    return [float(v).hex() for v in np.asarray(a, dtype=np.float64)]


def main():
    if oracle.ref() is None:
        sys.exit("oracle/_ref/libhnref.so is not built (make -C oracle ref)")
    write_lp_small(os.path.join(MPS_DIR, "lp_small.mps"))
    out = {}
    for name in sorted(os.listdir(MPS_DIR)):
        if not name.endswith(".mps"):
            continue
        text = open(os.path.join(MPS_DIR, name), "rb").read()
        for fmt in (-1, 0, 1):
            r = oracle.ref_mps(text, fmt)
            out[f"{name}:{fmt}"] = {
                "m": r["m"], "n": r["n"], "maximize": r["maximize"], "success": r["success"],
                "warnings": r["warnings"], "name": r["name"], "row_names": r["row_names"],
                "col_names": r["col_names"], "rp": [int(v) for v in r["rp"]], "ci": [int(v) for v in r["ci"]],
                "val": hx(r["val"]), "c": hx(r["c"]), "rhs": hx(r["rhs"]), "sense": [int(v) for v in r["sense"]],
                "lb": hx(r["lb"]), "ub": hx(r["ub"]), "range_lo": hx(r["range_lo"]), "range_hi": hx(r["range_hi"]),
                "vtype": [int(v) for v in r["vtype"]]}
    with open(OUT, "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)
    print(f"{len(out)} cases -> {OUT}")


if __name__ == "__main__":
    main()
