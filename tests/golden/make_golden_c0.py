"""Golden result of the reference IPM on the m=2000, n=5000, 8 nonzeros/column
LP (seed 0), crossover off: InteriorPointSolver::solve takes ~5 minutes here,
so the result is stored once (tests/golden/reference_ipm_c0.json).
Run from the repo root where oracle/_ref is built."""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "indigenous-cpu-gpu-optimization-engine-for-indian-industry_b200"))
import lpgen  # noqa: E402
import oracle as O  # noqa: E402

if __name__ == "__main__":
    out = {}
    for seed in (0,):
        lp = lpgen.lp_uniform(2000, 5000, 8, seed)
        r = O.ref_ipm_solve(lp)
        out[f"lp_uniform_2000_5000_8_seed{seed}"] = {"status": r["status"], "objective": r["objective"],
                                                      "iterations": r["iterations"], "time_ms": r["time_ms"]}
        print(out, flush=True)
    json.dump(out, open(os.path.join(HERE, "reference_ipm_c0.json"), "w"), indent=1)
