"""Writes tests/golden/mps_reference.json and tests/golden/lp_reference.json:
the reference's own readers (model::MPSParser / model::LPParser
::parse_string, compiled into oracle/_ref) run on every
tests/golden/mps/*.mps file (in the layout it detects and in both forced
layouts) and every tests/golden/lp/*.lp file. Doubles are stored as
float.hex strings (bit-exact). Also writes the generated instances
lp_small.mps and lp_small.lp (seeded LPs of the C0 generator, with repeated
and cancelling coefficients in the MPS one) before reading them.

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
LP_DIR = os.path.join(ROOT, "tests", "golden", "lp")
OUT = os.path.join(ROOT, "tests", "golden", "mps_reference.json")
OUT_LP = os.path.join(ROOT, "tests", "golden", "lp_reference.json")


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


def write_lp_small_lp(path):
    lp = lpgen.lp_uniform(80, 200, 5, seed=79)
    rp, ci, val = lp["rp"], lp["ci"], lp["val"]
    obj = " + ".join(f"{float(lp['c'][j])!r} v{j}" for j in range(lp["n"]))
    lines = ["Minimize", " obj: " + obj, "Subject To"]
    for i in range(lp["m"]):
        terms = " ".join(("- " if v < 0 else "+ ") + f"{abs(float(v))!r} v{int(j)}"
                         for j, v in zip(ci[rp[i]:rp[i + 1]], val[rp[i]:rp[i + 1]]))
        lines.append(f" r{i}: {terms} = {float(lp['b'][i])!r}")
    lines += ["Bounds"] + [f" v{j} <= {10 + j % 5}" for j in range(0, lp["n"], 4)] + ["End"]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def record(r):
    return {"m": r["m"], "n": r["n"], "maximize": r["maximize"], "success": r["success"],
            "errors": int(r.get("errors", 0)), "warnings": r["warnings"], "name": r["name"],
            "row_names": r["row_names"], "col_names": r["col_names"], "rp": [int(v) for v in r["rp"]],
            "ci": [int(v) for v in r["ci"]], "val": hx(r["val"]), "c": hx(r["c"]), "rhs": hx(r["rhs"]),
            "sense": [int(v) for v in r["sense"]], "lb": hx(r["lb"]), "ub": hx(r["ub"]),
            "range_lo": hx(r["range_lo"]), "range_hi": hx(r["range_hi"]), "vtype": [int(v) for v in r["vtype"]]}


def hx(a):
    return [float(v).hex() for v in np.asarray(a, dtype=np.float64)]


def main():
    if oracle.ref() is None:
        sys.exit("oracle/_ref/libhnref.so is not built (make -C oracle ref)")
    write_lp_small(os.path.join(MPS_DIR, "lp_small.mps"))
    write_lp_small_lp(os.path.join(LP_DIR, "lp_small.lp"))
    out = {}
    for name in sorted(os.listdir(MPS_DIR)):
        if name.endswith(".mps"):
            text = open(os.path.join(MPS_DIR, name), "rb").read()
            for fmt in (-1, 0, 1):
                out[f"{name}:{fmt}"] = record(oracle.ref_mps(text, fmt))
    with open(OUT, "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)
    out_lp = {}
    for name in sorted(os.listdir(LP_DIR)):
        if name.endswith(".lp"):
            out_lp[name] = record(oracle.ref_mps(open(os.path.join(LP_DIR, name), "rb").read(), lp_format=True))
    with open(OUT_LP, "w") as f:
        json.dump(out_lp, f, indent=0, sort_keys=True)
    print(f"{len(out)} MPS cases -> {OUT}, {len(out_lp)} LP cases -> {OUT_LP}")


if __name__ == "__main__":
    main()
