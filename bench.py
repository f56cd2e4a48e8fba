"""Benchmark of the FP64 sparse hot path under HyperNova's IPM on B200.

Workload (one "step" = one IPM iteration's sparse device work on the
m=200,000 x n=500,000 LP with Zipf(1.5) column counts at ~5.2M nonzeros,
scaled the way HyperNova's IPM scales it):
    y  = A x - b        (autotuned SpMV path, residual epilogue)
    t  = A^T lam        (SpMV on the device-built A^T)
    N  = A diag(D) A^T + dyn_reg I   (fixed-pattern assembly, nnz(N) ~ 9.7e8)
    x^T z, ||y||_inf, ||t||_inf      (deterministic reductions)
The metric is algorithmic GB/s of the whole step (bytes each kernel must
move by the formulas printed in `kernels`), measured with CUDA events on the
launching stream. `e2e` repeats the step through the same C ABI with the
inputs copied in from pinned host memory and the results -- y, t, the
scalars and the 7.8 GB of normal-matrix values the host factorisation reads
-- copied back inside the timed region. The step writes the 11.6 GB normal matrix, so every step
streams far more than the 126 MB L2 (no separate flush needed).

--impl reference times the reference's own CPU code for the same step
(CPUBackend::spmv, the IPM's matvec_t and build_normal_equations, compiled
from the reference sources into oracle/_ref) on all host cores, each thread on
its own bounded sample of columns for the assembly.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "indigenous-cpu-gpu-optimization-engine-for-indian-industry_b200")
sys.path.insert(0, PKG)

METRIC = "LP solves/s at 1e-8 KKT, batched+warm vs plain IPM on 1 B200; SpMV GB/s vs HBM"
WORKLOAD = "ipm-iteration sparse path, LP m=200000 n=500000 Zipf(1.5) cols nnz~5.2M (scaled standard form)"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock and throttle reasons sampled during the timed region: NVML
    queries every 10 ms (read-only), or nvidia-smi every 200 ms when NVML
    cannot be queried. The NVML handle and the reasons call are probed in
    start(), before the timed region, so a failing call falls back to
    nvidia-smi from the first sample on."""

    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int):
        self.index = index
        self.samples = []  # (sm MHz, max sm MHz, [reason flags in NAMES order])
        self.source = None
        self.note = None
        self._stop = threading.Event()
        self._t = None

    def _nvml_probe(self):
        import pynvml as nv

        nv.nvmlInit()
        h = nv.nvmlDeviceGetHandleByIndex(self.index)
        mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        reasons = None
        for name in ("nvmlDeviceGetCurrentClocksEventReasons", "nvmlDeviceGetCurrentClocksThrottleReasons"):
            fn = getattr(nv, name, None)
            if fn is None:
                continue
            try:
                fn(h)
                reasons = fn
                break
            except Exception:
                continue
        if reasons is None:
            raise RuntimeError("no NVML clock-reasons call")
        bits = [getattr(nv, "nvmlClocksEventReasonHwSlowdown", 0x8),
                getattr(nv, "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
                getattr(nv, "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
                getattr(nv, "nvmlClocksEventReasonSwPowerCap", 0x4)]

        def sample():
            r = reasons(h)
            return (float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), mx, [bool(r & b) for b in bits])

        sample()
        return nv, sample

    def _smi_sample(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits"],
                             capture_output=True, text=True, timeout=5).stdout.strip()
        f = [x.strip() for x in out.split(",")]
        if len(f) == 6 and f[0].replace(".", "").isdigit() and f[1].replace(".", "").isdigit():
            return (float(f[0]), float(f[1]), [x.lower() == "active" for x in f[2:]])
        return None

    def start(self):
        nv = sample = None
        try:
            nv, sample = self._nvml_probe()
            self.source = "nvml"
        except Exception as e:  # no NVML binding or call: nvidia-smi
            self.source = "nvidia-smi"
            self.note = f"nvml: {type(e).__name__}: {e}"[:160]

        def run():
            while not self._stop.is_set():
                try:
                    v = sample() if sample else self._smi_sample()
                    if v:
                        self.samples.append(v)
                except Exception as e:
                    self.note = f"{self.source}: {type(e).__name__}: {e}"[:160]
                self._stop.wait(0.01 if sample else 0.2)
            if nv is not None:
                try:
                    nv.nvmlShutdown()
                except Exception:
                    pass

        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        if not self.samples:
            out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "source": self.source}
            if self.note:
                out["note"] = self.note
            return out
        sm = [s[0] for s in self.samples]
        reasons = sorted({self.NAMES[i] for s in self.samples for i in range(4) if s[2][i]})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(s[1] for s in self.samples),
                "reasons": reasons, "samples": len(self.samples), "source": self.source}


def dist_setup():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def make_inputs(seed: int, scale: int = 1):
    import lpgen

    lp = lpgen.scaled_problem(lpgen.lp_zipf(m=200_000 // scale, n=500_000 // scale, seed=seed,
                                            target_nnz=5_000_000 // scale))
    rng = np.random.default_rng(seed + 1)
    m, n = lp["m"], lp["n"]
    vec = {"x": rng.uniform(0.5, 2.0, n), "z": rng.uniform(0.5, 2.0, n), "lam": rng.standard_normal(m)}
    vec["D"] = vec["x"] / vec["z"]
    return lp, vec


PROFILE_TRAFFIC = {"ada_numeric": "profiles/ada_numeric_c1-5m.md"}


def profiled_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from its committed ncu summary (the
    `traffic_per_launch_bytes:` line), or None."""
    rel = PROFILE_TRAFFIC.get(kernel)
    if not rel or not os.path.exists(os.path.join(ROOT, rel)):
        return None, None
    for line in open(os.path.join(ROOT, rel)):
        if line.startswith("traffic_per_launch_bytes:"):
            return int(line.split(":")[1]), rel
    return None, None


def step_bytes(m, n, nnz, nnz_t, nnz_n):
    """Algorithmic bytes per kernel (int32 indices for A / A^T, int64 row pointer for N)."""
    return {
        "spmv_A": 12 * nnz + 4 * (m + 1) + 8 * n + 8 * m + 8 * m,   # + b read by the residual epilogue
        "spmv_At": 12 * nnz_t + 4 * (n + 1) + 8 * m + 8 * n,
        "ada_numeric": 12 * nnz + 8 * n + 12 * nnz_n + 8 * (m + 1),
        "reductions": 16 * n + 8 * m + 8 * n,
    }


def run_ours(args, rank, world, local):
    import torch

    import hnb200 as hn

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    torch.zeros(1, device=dev)
    hn.init(local)
    lp, vec = make_inputs(1000 + rank)
    m, n = lp["m"], lp["n"]
    A = hn.Csr(m, n, lp["rp"], lp["ci"], lp["val"])
    P = hn.Pattern(A)
    f64 = torch.float64
    x = torch.as_tensor(vec["x"], device=dev)
    z = torch.as_tensor(vec["z"], device=dev)
    lam = torch.as_tensor(vec["lam"], device=dev)
    D = torch.as_tensor(vec["D"], device=dev)
    b = torch.as_tensor(lp["b"], device=dev)
    y = torch.empty(m, dtype=f64, device=dev)
    t = torch.empty(n, dtype=f64, device=dev)
    nval = torch.empty(P.nnz, dtype=f64, device=dev)
    scal = torch.zeros(8, dtype=f64, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    names = ["spmv_A", "spmv_At", "reductions", "ada_numeric"]
    # one event pair per (step, kernel group): read after a single final sync,
    # so no step waits on the host and per-kernel times are pure device time
    ev = [{k: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for k in names}
          for _ in range(args.steps)]

    def step(evs=None):
        def mark(k, i):
            if evs is not None:
                evs[k][i].record(stream)

        mark("spmv_A", 0)
        A.residual(x, b, y, trans=0, stream=sp)  # y = A x - b
        mark("spmv_A", 1)
        mark("spmv_At", 0)
        A.spmv(lam, t, trans=1, stream=sp)  # t = A^T lam
        mark("spmv_At", 1)
        mark("reductions", 0)
        hn.dot(n, x, z, scal[0:1], sp)
        hn.nrm_inf(m, y, scal[1:2], sp)
        hn.nrm_inf(n, t, scal[2:3], sp)
        mark("reductions", 1)
        mark("ada_numeric", 0)
        P.numeric(D, 1e-8, nval, scal[3:4], sp)
        mark("ada_numeric", 1)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0, _ = hn.stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(args.steps):
        step(ev[i])
    e1.record(stream)
    torch.cuda.synchronize()
    l1, _ = hn.stats()
    ms_total = e0.elapsed_time(e1)
    clk = clocks.stop()
    kt = {k: sum(ev[i][k][0].elapsed_time(ev[i][k][1]) for i in range(args.steps)) / args.steps for k in names}
    ms = ms_total / args.steps
    if world > 1:
        tt = torch.tensor([ms], dtype=f64, device=dev)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        ms = tt.item()
    nb = step_bytes(m, n, A.nnz, A.nnz_t, P.nnz)
    total_bytes = sum(nb.values())
    value = world * total_bytes / (ms * 1e-3) / 1e9

    # ---- end to end through the C ABI with pinned host buffers ----
    hx = torch.as_tensor(vec["x"]).pin_memory()
    hz = torch.as_tensor(vec["z"]).pin_memory()
    hl = torch.as_tensor(vec["lam"]).pin_memory()
    hD = torch.as_tensor(vec["D"]).pin_memory()
    hy = torch.empty(m, dtype=f64).pin_memory()
    ht = torch.empty(n, dtype=f64).pin_memory()
    hs = torch.empty(8, dtype=f64).pin_memory()
    # the normal matrix's values go back to the host every step: the IPM's
    # host factorisation reads them each iteration (hn_ipm.cpp, as the
    # reference's build_normal_equations leaves N on the host)
    hN = torch.empty(P.nnz, dtype=f64).pin_memory()
    lib = hn.load()

    def e2e_step():
        for dst, src, nb_ in ((x, hx, 8 * n), (z, hz, 8 * n), (lam, hl, 8 * m), (D, hD, 8 * n)):
            hn.check(lib.hn_memcpy_h2d(dst.data_ptr(), src.data_ptr(), nb_, sp))
        step()
        for dst, src, nb_ in ((hy, y, 8 * m), (ht, t, 8 * n), (hs, scal, 64), (hN, nval, 8 * P.nnz)):
            hn.check(lib.hn_memcpy_d2h(dst.data_ptr(), src.data_ptr(), nb_, sp))

    for _ in range(max(1, args.warmup)):
        e2e_step()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    h2d = 8 * (3 * n + m)
    d2h = 8 * (m + n) + 64 + 8 * P.nnz

    # SpMV on the spec-literal large LP (Zipf(1.5) columns on [1, 2000], no
    # rescaling: ~17M nonzeros), alone, L2 flushed between launches
    lit = spmv_literal(args, dev, stream) if not args.no_literal else None

    # the batched IPM runs on every rank (sharded when there are several)
    batch_result = None if args.no_batch else batched_ipm(args.batch_k, args.batch_sample, rank, world)

    result = None
    if rank == 0:
        hbm, how = peaks()
        dom = max(kt, key=kt.get)
        achieved = nb[dom] / (kt[dom] * 1e-3) / 1e9
        traffic, traffic_src = profiled_traffic(dom)
        result = {
            "metric": METRIC, "value": round(value, 1), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded lpgen Zipf LP per rank)",
            "config": {"workload": WORKLOAD, "m": m, "n": n, "nnz": A.nnz, "nnz_N": P.nnz,
                       "l2": "inputs larger than L2 (each step writes the 11.6 GB normal matrix)",
                       "parallelism": f"replicas x{world} (independent LP per rank, no collective)"},
            "e2e": {"value": round(world * total_bytes / (e2e_ms * 1e-3) / 1e9, 1), "unit": "GB/s",
                    "ms_per_step": round(e2e_ms, 4), "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(l1 - l0),
            "kernels": {k: {"ms": round(kt[k], 4), "bytes": nb[k], "GB/s": round(nb[k] / (kt[k] * 1e-3) / 1e9, 1)}
                        for k in names},
            "roofline": {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 1), "peak": hbm,
                         "peak_source": how, "unit": "GB/s", "frac": round(achieved / hbm, 4), "traffic": traffic,
                         "traffic_source": traffic_src, "bytes_per_launch": nb[dom]},
            "clocks": clk,
        }
        if lit is not None:
            result["kernels"].update(lit)
        if not args.no_ipm:
            result["plain_ipm"] = plain_ipm()
        if batch_result is not None:
            result["batched_ipm"] = batch_result
        if not args.no_gnn:
            # the GNN warm start at reduced scale (the config's 20,000 training
            # and 4,096 evaluation LPs are the --only gnn mode)
            result["gnn_warm_small"] = gnn_warm(args.small_gnn, args.small_gnn, 500, 5000, 20, 256, plain_sample=6)
        if not args.no_cpu_baseline:
            result["cpu_baseline"] = cpu_baseline(lp, vec, threads=os.cpu_count() or 1, reps=1)
    return result


def spmv_literal(args, dev, stream):
    """y = A x and y = A^T x on the spec-literal LP (m 200k, n 500k, Zipf(1.5)
    column counts on [1, 2000] without rescaling, ~17M nonzeros, seed 1000),
    autotuned path, CUDA events around each launch, a 256 MB write between
    launches (cold L2), mean over the timed launches."""
    import torch

    import hnb200 as hn
    import lpgen

    lp = lpgen.lp_zipf(seed=1000, target_nnz=None)
    m, n = lp["m"], lp["n"]
    A = hn.Csr(m, n, lp["rp"], lp["ci"], lp["val"])
    sp = stream.cuda_stream
    flush = torch.empty(32 * 1024 * 1024, dtype=torch.float64, device=dev)
    out = {}
    for name, trans in (("spmv_A_c1_literal", 0), ("spmv_At_c1_literal", 1)):
        xin = torch.as_tensor(lp["y0"] if trans else lp["x0"], device=dev)
        yout = torch.empty(n if trans else m, dtype=torch.float64, device=dev)
        nbytes = (12 * A.nnz_t + 4 * (n + 1) + 8 * m + 8 * n) if trans else (12 * A.nnz + 4 * (m + 1) + 8 * n + 8 * m)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for _ in range(args.warmup):
            flush.zero_()
            A.spmv(xin, yout, trans=trans, stream=sp)
        for i in range(args.steps):
            flush.zero_()
            evs[i][0].record(stream)
            A.spmv(xin, yout, trans=trans, stream=sp)
            evs[i][1].record(stream)
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in evs) / args.steps
        out[name] = {"ms": round(ms, 4), "bytes": nbytes, "GB/s": round(nbytes / (ms * 1e-3) / 1e9, 1),
                     "nnz": A.nnz if not trans else A.nnz_t, "path": list(A.spmv_kind(trans))}
    A.close()
    return out


def plain_ipm():
    """One solve of the m=2000, n=5000, 8 nonzeros/column LP (seed 0) by the
    plain GPU IPM (crossover off), against the reference's stored result."""
    import hnb200 as hn
    import lpgen

    lp = lpgen.lp_uniform(2000, 5000, 8, 0)
    r = hn.lp_solve(lp)
    ref = None
    gp = os.path.join(ROOT, "tests", "golden", "reference_ipm_c0.json")
    if os.path.exists(gp):
        ref = json.load(open(gp))["lp_uniform_2000_5000_8_seed0"]
    out = {"lp": "m=2000 n=5000 8 nnz/col seed 0", "status": r["status_name"], "iterations": r["iterations"],
           "reference_rule_iterations": r["reference_iterations"], "relative_kkt": r["kkt"],
           "objective": r["objective"], "ms": round(r["time_ms"], 1), "solves_per_s": round(1e3 / r["time_ms"], 3),
           "factor_ms": round(r["factor_ms"], 1), "device_ms": round(r["device_ms"], 1),
           "host_threads": os.cpu_count()}
    if ref:
        out["reference"] = {"status": ref["status"], "objective": ref["objective"], "iterations": ref["iterations"],
                            "ms": round(ref["time_ms"], 1), "rel_obj_diff": abs(r["objective"] - ref["objective"]) /
                            (1.0 + abs(ref["objective"]))}
    return out


def batched_ipm(K: int, sample_per_stratum: int = 4, rank: int = 0, world: int = 1):
    """The 4096-LP batch (m log-uniform in [50, 2000], n = round(2.5 m),
    6 nonzeros per column, seeds 20000+i) through the batched GPU IPM, and the
    plain one-at-a-time GPU IPM on a seeded stratified sample of the same
    instances (8 log-size strata), extrapolated to the batch. Wall-clock
    times with the device synchronised on both sides; both include the
    host->device copies of the LPs and the device->host copies of the
    solutions. With several ranks the batch is sharded by LPT greedy over
    the ranks (shard.py: no data-path collective, one gather of the results)
    and timed as the max over ranks; the plain sample runs on rank 0."""
    import torch

    import hnb200 as hn
    import lpgen
    import shard

    sizes = lpgen.batch_sizes(K, seed=2000)
    lps = [lpgen.lp_uniform(int(m), int(round(2.5 * m)), 6, 20000 + i) for i, m in enumerate(sizes)]
    if world > 1:
        torch.distributed.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        def solve_part(part, **kw):
            res = hn.lp_solve_batch(part, **kw)
            res["kkt0"] = res["kkt"][:, 0]
            return res

        r = shard.solve_sharded(lps, solve_part, rank, world, keys=("status", "objective", "iterations", "kkt0"))
        torch.cuda.synchronize()
        wall_t = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(wall_t, op=torch.distributed.ReduceOp.MAX)
        if rank != 0:
            return None
        wall = float(wall_t.item())
        st = r["status"]
        return {"workload": f"{K} LPs, m log-uniform [50,2000], n=2.5m, 6 nnz/col (seeds 20000+i)",
                "ranks": world, "sharding": "LPT greedy on m^3/3 + nnz, one gather of the results",
                "instances_per_rank": [int(p.size) for p in r["parts"]], "batched_s": round(wall, 3),
                "batched_solves_per_s": round(K / wall, 1), "optimal": int((st == 1).sum()),
                "kkt_le_1e-8": int(((st == 1) & (r["kkt0"] <= 1e-8)).sum()), "kkt_max": float(np.nanmax(r["kkt0"])),
                "iterations_mean": round(float(np.mean(r["iterations"])), 2)}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = hn.lp_solve_batch(lps)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    st = r["status"]
    kkt = r["kkt"][:, 0]
    at_kkt = (st == 1) & (kkt <= 1e-8)
    # dense LDL^T work: one factorisation of m_i^3 / 3 multiply-adds per iteration of each instance
    factor_flops = float(np.sum(r["iterations"].astype(np.float64) * sizes.astype(np.float64) ** 3 * 2.0 / 3.0))
    # stratified plain sample
    edges = np.exp(np.linspace(np.log(50), np.log(2000) + 1e-9, 9))
    rng = np.random.default_rng(7)
    est, matched, sampled, plain_iters, plain_kkt_ok = 0.0, 0, 0, [], 0
    for a, b in zip(edges[:-1], edges[1:]):
        idx = np.nonzero((sizes >= a) & (sizes < b))[0]
        if idx.size == 0 or sample_per_stratum == 0:
            continue
        pick = rng.choice(idx, size=min(sample_per_stratum, idx.size), replace=False)
        times = []
        for i in pick:
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            p = hn.lp_solve(lps[i])
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t1)
            plain_iters.append(p["iterations"])
            sampled += 1
            rel = abs(p["objective"] - r["objective"][i]) / (1.0 + abs(p["objective"]))
            matched += int(p["status"] == st[i] == 1 and rel <= 1e-8)
            plain_kkt_ok += int(p["status"] == 1 and p["kkt"] <= 1e-8)
        est += float(np.mean(times)) * idx.size
    return {"workload": f"{K} LPs, m log-uniform [50,2000], n=2.5m, 6 nnz/col (seeds 20000+i)",
            "rows": int(sizes.sum()), "batched_s": round(wall, 3), "batched_solves_per_s": round(K / wall, 1),
            "optimal": int((st == 1).sum()), "kkt_le_1e-8": int(at_kkt.sum()),
            "batched_solves_per_s_at_1e-8_kkt": round(int(at_kkt.sum()) / wall, 1),
            "kkt_max": float(np.nanmax(kkt)), "kkt_median": float(np.nanmedian(kkt)),
            "iterations_max": int(r["stats"]["iterations"]),
            "iterations_mean": round(float(r["iterations"].mean()), 2),
            "reference_rule_iterations_mean": round(float(r["reference_iterations"].mean()), 2),
            "factor_ms": round(r["stats"]["factor_ms"], 1), "solve_ms": round(r["stats"]["solve_ms"], 1),
            "forms_ms": round(r["stats"]["forms_ms"], 1), "setup_ms": round(r["stats"]["setup_ms"], 1),
            "total_ms": round(r["stats"]["total_ms"], 1),
            "factor_fp64_tflops": round(factor_flops / (r["stats"]["factor_ms"] * 1e-3) / 1e12, 2),
            "plain_gpu_s_extrapolated": round(est, 2) if sampled else None,
            "plain_gpu_solves_per_s_extrapolated": round(K / est, 2) if sampled else None,
            "speedup_vs_plain_gpu": round(est / wall, 2) if sampled else None,
            "plain_sample": {"instances": sampled, "per_stratum": sample_per_stratum,
                             "matching_status_and_objective_1e-8": matched, "kkt_le_1e-8": plain_kkt_ok,
                             "iterations_mean": round(float(np.mean(plain_iters)), 2) if sampled else None}}


def bb_batch(K: int, chunk: int, sample: int = 2):
    """Branch-and-bound style batch: one base LP (m=5000, n=12000, 8 nonzeros
    per column, seed 3000) and K node relaxations (lpgen.bb_nodes, seed 3000),
    each warm-started from the base LP's barrier solution (primal and dual
    estimate), solved by the batched GPU IPM in chunks of `chunk` nodes (the
    dense normal-matrix factors of a chunk share the device); the plain GPU
    IPM on `sample` nodes, extrapolated."""
    import torch

    import hnb200 as hn
    import lpgen

    base = lpgen.lp_uniform(5000, 12000, 8, 3000)
    nodes = lpgen.bb_nodes(base, K)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r0 = hn.lp_solve(base)
    base_s = time.perf_counter() - t0
    status, obj, iters, used, kkt = [], [], [], [], []
    t0 = time.perf_counter()
    for c0 in range(0, K, chunk):
        part = nodes[c0:c0 + chunk]
        r = hn.lp_solve_batch([base] * len(part), lbs=[a for a, _ in part], ubs=[b for _, b in part],
                              x0s=[r0["x"]] * len(part), y0s=[r0["y"]] * len(part))
        status.append(r["status"])
        obj.append(r["objective"])
        iters.append(r["iterations"])
        used.append(r["warm_used"])
        kkt.append(r["kkt"][:, 0])
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    status, obj, iters, used, kkt = map(np.concatenate, (status, obj, iters, used, kkt))
    pt, matched = [], 0
    for i in range(sample):
        t1 = time.perf_counter()
        p = hn.lp_solve(base, lb=nodes[i][0], ub=nodes[i][1])
        torch.cuda.synchronize()
        pt.append(time.perf_counter() - t1)
        matched += int(p["status"] == status[i] and abs(p["objective"] - obj[i]) / (1 + abs(p["objective"])) <= 1e-8)
    est = float(np.mean(pt)) * K
    return {"workload": f"B&B batch: base LP m=5000 n=12000 8 nnz/col (seed 3000), {K} node relaxations "
                        f"(1-40 bound changes each), warm-started from the base solution, chunks of {chunk}",
            "base_solve_s": round(base_s, 2), "base_iterations": r0["iterations"],
            "batched_s": round(wall, 2), "batched_solves_per_s": round(K / wall, 2),
            "status_counts": {int(k): int(v) for k, v in zip(*np.unique(status, return_counts=True))},
            "warm_used": int(used.sum()), "iterations_mean": round(float(iters.mean()), 2),
            "kkt_le_1e-8": int(((status == 1) & (kkt <= 1e-8)).sum()), "kkt_median": float(np.nanmedian(kkt)),
            "plain_gpu_s_extrapolated": round(est, 1), "plain_gpu_solves_per_s_extrapolated": round(K / est, 3),
            "speedup_vs_plain_gpu": round(est / wall, 2), "plain_sample": {"instances": sample, "matching": matched}}


def gnn_warm(n_train: int, n_eval: int, mlo: int, mhi: int, epochs: int, chunk: int, plain_sample: int = 8):
    # n_eval LPs: cold and warm batched solves; plain_sample of them by the plain GPU IPM
    """GNN warm start: LPs of the m=2000 generator with m log-uniform in
    [mlo, mhi] and n = round(2.5 m), 8 nonzeros per column. Training LPs
    (seeds 4,000,000 + i) are labelled by the batched GPU IPM (its primal
    and dual estimate), the network is trained on the GPU (gnn.py), and
    fresh LPs (seeds 1,000,000 + i) are solved by the batched GPU IPM from
    the default start and from the network's prediction (inference time
    included), and a sample by the plain one-at-a-time GPU IPM."""
    import torch

    import gnn
    import hnb200 as hn
    import lpgen

    def gen(count, seed0):
        rng = np.random.default_rng(seed0)
        sizes = np.round(np.exp(rng.uniform(np.log(mlo), np.log(mhi), count))).astype(int)
        return [lpgen.lp_uniform(int(m), int(round(2.5 * m)), 8, seed0 + i) for i, m in enumerate(sizes)]

    infer = [0.0]

    def batched(lps, warm=None):
        out = {"status": [], "objective": [], "iterations": [], "warm_used": [], "kkt": [], "x": [], "y": [], "s": []}
        for c0 in range(0, len(lps), chunk):
            part = lps[c0:c0 + chunk]
            kw = {}
            if warm is not None:
                ti = time.perf_counter()
                preds = gnn.predict(warm, gnn.Batch(part))
                torch.cuda.synchronize()
                infer[0] += time.perf_counter() - ti
                kw = {"x0s": [p[0] for p in preds], "y0s": [p[1] for p in preds], "s0s": [p[2] for p in preds],
                      "warm_floor": gnn.WARM_FLOOR}
            r = hn.lp_solve_batch(part, **kw)
            for k in ("status", "objective", "iterations", "warm_used"):
                out[k].append(r[k])
            out["kkt"].append(r["kkt"][:, 0])
            for k, lp in enumerate(part):
                c0_, c1_ = r["col_off"][k], r["col_off"][k + 1]
                r0_, r1_ = r["row_off"][k], r["row_off"][k + 1]
                out["x"].append(r["x"][c0_:c1_])
                out["y"].append(r["y"][r0_:r1_])
                out["s"].append(r["s"][c0_:c1_])
        for k in ("status", "objective", "iterations", "warm_used", "kkt"):
            out[k] = np.concatenate(out[k])
        return out

    train_lps = gen(n_train, 4_000_000)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lab = batched(train_lps)
    label_s = time.perf_counter() - t0
    print(json.dumps({"gnn_progress": "labelled", "train": n_train, "label_s": round(label_s, 1)}), file=sys.stderr,
          flush=True)
    keep = [i for i in range(n_train) if lab["status"][i] == 1]
    batches = []
    for j in range(0, len(keep), 8):
        ids = keep[j:j + 8]
        batches.append(gnn.Batch([train_lps[i] for i in ids], [(lab["x"][i], lab["y"][i], lab["s"][i]) for i in ids]))
    model = gnn.Model(seed=0)
    t0 = time.perf_counter()
    losses = gnn.train(model, batches, epochs=epochs, lr=1e-3)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    del batches
    print(json.dumps({"gnn_progress": "trained", "train_s": round(train_s, 1),
                      "loss_first_last": [losses[0], losses[-1]]}), file=sys.stderr, flush=True)

    eval_lps = gen(n_eval, 1_000_000)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    cold = batched(eval_lps)
    torch.cuda.synchronize()
    cold_s = time.perf_counter() - t0
    print(json.dumps({"gnn_progress": "cold", "cold_s": round(cold_s, 2),
                      "iterations_mean_cold": float(cold["iterations"].mean())}), file=sys.stderr, flush=True)
    t0 = time.perf_counter()
    warm = batched(eval_lps, warm=model)
    torch.cuda.synchronize()
    warm_s = time.perf_counter() - t0
    same = (cold["status"] == warm["status"]) & (np.abs(cold["objective"] - warm["objective"]) <=
                                                  1e-8 * (1 + np.abs(cold["objective"])))
    # the batched factorisation's work is ~ iterations x m^3 per instance
    m3 = np.array([float(lp["m"]) ** 3 for lp in eval_lps])
    work_ratio = float((warm["iterations"] * m3).sum() / (cold["iterations"] * m3).sum())
    pt = []
    for i in range(min(plain_sample, n_eval)):
        t1 = time.perf_counter()
        hn.lp_solve(eval_lps[i])
        torch.cuda.synchronize()
        pt.append(time.perf_counter() - t1)
    plain_est = float(np.mean(pt)) * n_eval
    return {"workload": f"m=2000-generator LPs, m log-uniform [{mlo},{mhi}], n=2.5m, 8 nnz/col; "
                        f"train {n_train} (seeds 4e6+i), eval {n_eval} fresh (seeds 1e6+i)",
            "label_s": round(label_s, 1), "train_s": round(train_s, 1), "epochs": epochs,
            "loss_first_last": [round(losses[0], 4), round(losses[-1], 4)],
            "cold_batched_s": round(cold_s, 2), "cold_batched_solves_per_s": round(n_eval / cold_s, 2),
            "warm_batched_s": round(warm_s, 2), "warm_batched_solves_per_s": round(n_eval / warm_s, 2),
            "warm_inference_s": round(infer[0], 2),
            "iterations_mean_cold": round(float(cold["iterations"].mean()), 2),
            "iterations_mean_warm": round(float(warm["iterations"].mean()), 2),
            "factor_work_warm_over_cold": round(work_ratio, 4),
            "warm_used": int(warm["warm_used"].sum()), "optimal_cold": int((cold["status"] == 1).sum()),
            "optimal_warm": int((warm["status"] == 1).sum()),
            "kkt_le_1e-8_cold": int(((cold["status"] == 1) & (cold["kkt"] <= 1e-8)).sum()),
            "kkt_le_1e-8_warm": int(((warm["status"] == 1) & (warm["kkt"] <= 1e-8)).sum()),
            "same_status_and_objective_1e-8": int(same.sum()),
            "plain_gpu_solves_per_s_extrapolated": round(n_eval / plain_est, 3),
            "warm_batched_vs_plain_gpu": round(plain_est / warm_s, 2)}


def pricing(A, m, n, steps, warmup, flush):
    """Device simplex pricing on the bench LP: reduced costs (A^T SpMV with the
    rc = c - A^T y epilogue), a Devex update (A^T u, masked max, weights),
    the entering choice (Bland; ranked top-1 and top-16) and a 16-column
    gather; per call time (CUDA events, L2 flushed) and algorithmic bytes."""
    import torch

    import hnb200 as hn

    rng = np.random.default_rng(5)
    dev = "cuda"
    y = torch.as_tensor(rng.standard_normal(m), device=dev)
    u = torch.as_tensor(rng.standard_normal(m), device=dev)
    cost = torch.as_tensor(rng.standard_normal(n), device=dev)
    nb = np.arange(n, dtype=np.int32)
    nb[rng.choice(n, m, replace=False)] = -1
    nonbasis = torch.as_tensor(nb, device=dev)
    art = torch.zeros(n, dtype=torch.uint8, device=dev)
    rc = torch.empty(n, dtype=torch.float64, device=dev)
    w = torch.ones(n, dtype=torch.float64, device=dev)
    alpha = torch.empty(n, dtype=torch.float64, device=dev)
    out = torch.empty(17, dtype=torch.int64, device=dev)
    cols = torch.as_tensor(rng.choice(n, 16, replace=False).astype(np.int64), device=dev)
    colbuf = torch.empty((16, m), dtype=torch.float64, device=dev)
    spmv_t = 12 * A.nnz_t + 4 * (n + 1) + 8 * m
    ops = {
        "reduced_costs": (lambda: hn.price_reduced_costs(A, y, cost, rc), spmv_t + 16 * n),
        "devex_update": (lambda: hn.price_devex_update(A, u, nonbasis, w, alpha), spmv_t + 8 * n + 2 * (12 * n)),
        "select_bland": (lambda: hn.price_select(n, rc, w, nonbasis, art, out, rule=hn.PRICE_BLAND), 21 * n),
        "select_ranked_k1": (lambda: hn.price_select(n, rc, w, nonbasis, art, out, k=1), 3 * 21 * n),
        "select_ranked_k16": (lambda: hn.price_select(n, rc, w, nonbasis, art, out, k=16), 33 * 21 * n),
        "columns_k16": (lambda: hn.price_columns(A, cols, colbuf), 16 * 8 * m),
    }
    res = {}
    for name, (fn, nbytes) in ops.items():
        for _ in range(warmup):
            flush.zero_()
            fn()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            flush.zero_()
            evs[i][0].record()
            fn()
            evs[i][1].record()
        torch.cuda.synchronize()
        ms = sorted(a.elapsed_time(b) for a, b in evs)[steps // 2]
        res[name] = {"us": round(ms * 1e3, 2), "bytes": int(nbytes), "GB/s": round(nbytes / (ms * 1e-3) / 1e9, 1)}
    return {"workload": f"simplex pricing on the LP m={m} n={n} nnz={A.nnz} (m basic columns)", **res}


def gnn_layer(steps, warmup, rows=1 << 20):
    """One 128 -> 64 GNN layer over `rows` rows (X = [X1 | X2], FP32, 512 MB
    at 2^20 rows): the tcgen05 kernel and the mma.sync kernel, per call time
    (CUDA events; the input exceeds L2), bytes (X read, Y written) and flops;
    and its backward (hn_gnn_linear_bwd: G = dY relu'(Y), dX = G W^T and
    dW = X^T G on the tcgen05 kernels) with bytes Y, dY read, G written and
    read twice, dX written, X read."""
    import torch

    import hnb200 as hn

    g = torch.Generator(device="cuda").manual_seed(3)
    X1 = torch.randn((rows, 64), generator=g, device="cuda")
    X2 = torch.randn((rows, 64), generator=g, device="cuda")
    W = torch.randn(128 * 64, generator=g, device="cuda") / 128 ** 0.5
    b = torch.zeros(64, device="cuda")
    Wt = torch.empty(128 * 64, dtype=torch.bfloat16, device="cuda")
    Wb = torch.empty(128 * 64, dtype=torch.bfloat16, device="cuda")
    Y = torch.empty((rows, 64), device="cuda")
    dY = torch.randn((rows, 64), generator=g, device="cuda")
    G = torch.empty((rows, 64), device="cuda")
    dX = torch.empty((rows, 128), device="cuda")
    dW = torch.empty(128 * 64, device="cuda")
    db = torch.empty(64, device="cuda")
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    scratch = torch.empty(sms * (128 * 64 + 64), device="cuda")
    lib = hn.load()
    hn.check(lib.hn_gnn_cast_weights(128, W.data_ptr(), Wt.data_ptr(), Wb.data_ptr(), None))
    calls = {
        "tcgen05": lambda: hn.check(lib.hn_gnn_linear_umma(rows, 64, 64, X1.data_ptr(), X2.data_ptr(), Wt.data_ptr(),
                                                           b.data_ptr(), 1, Y.data_ptr(), None)),
        "mma_sync": lambda: hn.check(lib.hn_gnn_linear(rows, 64, 64, X1.data_ptr(), X2.data_ptr(), Wt.data_ptr(), 64,
                                                       b.data_ptr(), 1, Y.data_ptr(), None)),
        "backward_tcgen05": lambda: hn.check(lib.hn_gnn_linear_bwd(
            rows, 64, 64, X1.data_ptr(), X2.data_ptr(), Wb.data_ptr(), Y.data_ptr(), dY.data_ptr(), 1, G.data_ptr(),
            dX.data_ptr(), dW.data_ptr(), db.data_ptr(), scratch.data_ptr(), scratch.numel(), None)),
    }
    fwd_bytes, fwd_flops = rows * (128 * 4 + 64 * 4), 2 * rows * 128 * 64
    work = {"tcgen05": (fwd_bytes, fwd_flops), "mma_sync": (fwd_bytes, fwd_flops),
            "backward_tcgen05": (rows * 4 * (64 * 3 + 64 * 2 + 128 + 128), 2 * 2 * rows * 128 * 64)}
    res = {"workload": f"GNN layer [X1 | X2] ({rows} x 128, FP32) x W (128 x 64, BF16) + b, ReLU, and its backward"}
    hn.check(lib.hn_gnn_check(None))
    for name, fn in calls.items():
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        ms = sorted(ts)[steps // 2]
        hn.check(lib.hn_gnn_check(None))
        nbytes, flops = work[name]
        res[name] = {"us": round(ms * 1e3, 1), "GB/s": round(nbytes / (ms * 1e-3) / 1e9, 1),
                     "TFLOP/s": round(flops / (ms * 1e-3) / 1e12, 2)}
    return res


def _mps_text(lp: dict, name: str) -> bytes:
    """Free-layout MPS of an LP dict (EQ rows, x >= 0), column by column."""
    m, n = lp["m"], lp["n"]
    rp, ci, val = lp["rp"], lp["ci"], lp["val"]
    order = np.argsort(ci, kind="stable")
    rows = np.repeat(np.arange(m), np.diff(rp.astype(np.int64)))[order]
    cols = ci[order].astype(np.int64)
    vals = val[order]
    out = [f"NAME {name}", "ROWS", " N obj"] + [f" E r{i}" for i in range(m)] + ["COLUMNS"]
    starts = np.searchsorted(cols, np.arange(n + 1))
    for j in range(n):
        out.append(f"    v{j} obj {float(lp['c'][j])!r}")
        out.extend(f"    v{j} r{i} {a!r}" for i, a in zip(rows[starts[j]:starts[j + 1]].tolist(),
                                                        vals[starts[j]:starts[j + 1]].tolist()))
    out.append("RHS")
    out.extend(f"    rhs r{i} {b!r}" for i, b in enumerate(lp["b"].tolist()))
    out.append("ENDATA")
    return ("\n".join(out) + "\n").encode()


def mps_io(sample_m: int = 2000):
    """MPS reading into device CSR. (1) The product reader (hn_mps, host C++)
    and the reference's MPSParser::parse_string on the same text: a seeded
    LP of the C0 generator (m = sample_m, n = 2.5 m, 6 nonzeros per column).
    (2) The large LP (m = 200k, n = 500k, 5.16M nonzeros) through the
    product reader and hn_csr_create_coo; the reference's parser looks rows
    up by linear search (quadratic in the row count) and is not run there.
    (3) hn_csr_create_coo against the reference's SparseMatrix::from_triplets
    on the large LP's triplets. Wall-clock, best of 3."""
    import ctypes as C

    import torch

    import hnb200 as hn
    import lpgen

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    def reader_ms(text):
        best = float("inf")
        for _ in range(3):
            h = C.c_void_p()
            t0 = time.perf_counter()
            hn.host_check(hn.host().hn_mps_read_string(text, len(text), -1, C.byref(h)))
            best = min(best, (time.perf_counter() - t0) * 1e3)
            hn.host().hn_mps_free(h)
        return best

    res = {"workload": "MPS text -> device CSR"}
    small = lpgen.lp_uniform(sample_m, int(2.5 * sample_m), 6, seed=1000)
    t_small = _mps_text(small, "C0")
    ref_ms = None
    if oracle.ref() is not None:
        ref_ms = min(oracle.ref_mps_parse_ms(t_small) for _ in range(3))
    ours = reader_ms(t_small)
    res["c0_sample"] = {"m": small["m"], "n": small["n"], "nnz": int(small["rp"][-1]), "bytes": len(t_small),
                        "reader_ms": round(ours, 2), "reference_parser_ms": None if ref_ms is None else round(ref_ms, 2),
                        "speedup": None if ref_ms is None else round(ref_ms / ours, 1)}
    big = lpgen.lp_zipf()
    t_big = _mps_text(big, "C1")
    ours_big = reader_ms(t_big)
    h = C.c_void_p()
    hn.host_check(hn.host().hn_mps_read_string(t_big, len(t_big), -1, C.byref(h)))
    nt = C.c_int64()
    hn.host_check(hn.host().hn_mps_shape(h, None, None, C.byref(nt), None))
    tr, tc, tv = np.empty(nt.value, np.int64), np.empty(nt.value, np.int64), np.empty(nt.value)
    hn.host_check(hn.host().hn_mps_arrays(h, hn._p(tr, C.c_int64), hn._p(tc, C.c_int64), hn._p(tv, C.c_double),
                                          None, None, None, None, None, None, None, None))
    hn.host().hn_mps_free(h)
    m, n = big["m"], big["n"]
    coo = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        A = hn.Csr.from_coo(m, n, tr, tc, tv, transpose=False, autotune=False)
        torch.cuda.synchronize()
        coo.append((time.perf_counter() - t0) * 1e3)
        A.close()
    ref_ft = None
    if oracle.ref() is not None:
        t0 = time.perf_counter()
        oracle.ref_from_triplets(m, n, tr, tc, tv)
        ref_ft = (time.perf_counter() - t0) * 1e3
    res["c1_5m"] = {"m": m, "n": n, "nnz": int(nt.value), "bytes": len(t_big), "reader_ms": round(ours_big, 1),
                    "reader_MB/s": round(len(t_big) / (ours_big * 1e-3) / 1e6, 1),
                    "coo_to_device_csr_ms": round(min(coo), 2),
                    "reference_from_triplets_ms": None if ref_ft is None else round(ref_ft, 1)}
    return res


def run_only(args, local):
    """Single kernel group on the same LP (profiling aid). spmv / spmv_t flush
    L2 between launches by writing a 256 MB buffer; ada streams 11.6 GB."""
    import torch

    import hnb200 as hn

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    torch.zeros(1, device=dev)
    hn.init(local)
    if args.only == "bb":
        return bb_batch(args.bb_k, args.bb_chunk)
    if args.only == "batch":
        return batched_ipm(args.batch_k, args.batch_sample)
    if args.only == "gnn_layer":
        return gnn_layer(args.steps, args.warmup)
    if args.only == "mps":
        return mps_io()
    if args.only == "gnn":
        return gnn_warm(args.gnn_train, args.gnn_eval, args.gnn_mlo, args.gnn_mhi, args.gnn_epochs, args.gnn_chunk)
    if args.literal:
        import lpgen

        lp = lpgen.lp_zipf(seed=1000, target_nnz=None)
        vec = {"x": lp["x0"], "lam": lp["y0"], "D": np.ones(lp["n"])}
    else:
        lp, vec = make_inputs(1000, args.scale)
    m, n = lp["m"], lp["n"]
    A = hn.Csr(m, n, lp["rp"], lp["ci"], lp["val"])
    if args.spmv_kind >= 0:
        A.set_spmv_kind(args.spmv_kind, args.spmv_t, trans=0)
        A.set_spmv_kind(args.spmv_kind, args.spmv_t, trans=1)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    flush = torch.empty(32 * 1024 * 1024, dtype=torch.float64, device=dev)
    if args.only == "price":
        return pricing(A, m, n, args.steps, args.warmup, flush)
    if args.only == "ada":
        P = hn.Pattern(A, layout=None if args.ada_layout < 0 else args.ada_layout)
        D = torch.as_tensor(vec["D"], device=dev)
        nval = torch.empty(P.nnz, dtype=torch.float64, device=dev)
        nbytes = step_bytes(m, n, A.nnz, A.nnz_t, P.nnz)["ada_numeric"]
        fn = lambda: P.numeric(D, 1e-8, nval, None, sp)  # noqa: E731
    else:
        trans = 1 if args.only == "spmv_t" else 0
        xin = torch.as_tensor(vec["lam"] if trans else vec["x"], device=dev)
        yout = torch.empty(n if trans else m, dtype=torch.float64, device=dev)
        nbytes = step_bytes(m, n, A.nnz, A.nnz_t, 0)["spmv_At" if trans else "spmv_A"] - (0 if trans else 8 * m)
        fn = lambda: A.spmv(xin, yout, trans=trans, stream=sp)  # noqa: E731
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for _ in range(args.warmup):
        flush.zero_()
        fn()
    for i in range(args.steps):
        flush.zero_()
        evs[i][0].record(stream)
        fn()
        evs[i][1].record(stream)
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in evs) / args.steps
    hbm, how = peaks()
    extra = {}
    if args.only == "ada":
        extra["layout"] = P.mode()[0]
    else:
        extra["path"] = list(A.spmv_kind(1 if args.only == "spmv_t" else 0))
    return {"only": args.only, "scale": args.scale, "literal": args.literal, **extra, "m": m, "n": n, "nnz": A.nnz,
            "ms": round(ms, 4), "bytes": nbytes, "GB/s": round(nbytes / (ms * 1e-3) / 1e9, 1),
            "frac_of_" + how + "_hbm": round(nbytes / (ms * 1e-3) / 1e9 / hbm, 4)}


def cpu_baseline(lp, vec, threads: int, reps: int):
    """Reference CPU code on the same step, bounded sample (see module doc)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    if O.ref() is None:
        return {"value": None, "unit": "GB/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref not built"}
    m, n = lp["m"], lp["n"]
    ns = 8000 * threads  # columns fed to build_normal_equations, split over the threads
    secs, trip, nnzn = O.ref_step_sample(lp, vec["x"], vec["lam"], vec["D"], ns, threads, reps)
    nnz = len(lp["ci"])
    cols = np.bincount(lp["ci"], minlength=n)
    nnz_s = int(cols[:ns].sum())
    per = (12 * nnz + 4 * (m + 1) + 16 * n + 8 * m) + (12 * nnz + 4 * (n + 1) + 16 * m)  # spmv + matvec_t
    bytes_total = reps * (threads * per + 12 * nnz_s + 8 * ns + 12 * nnzn + 8 * (m + 1) * threads)
    return {"value": round(bytes_total / secs / 1e9, 3), "unit": "GB/s", "cores": threads, "kind": "reference",
            "seconds": round(secs, 3),
            "sample": f"{threads} threads x {reps} pass: full A x and A^T lam each, build_normal_equations on "
                      f"{ns} of {n} columns ({trip} triplets, nnz(N) {nnzn})"}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    lp, vec = make_inputs(1000)
    threads = os.cpu_count() or 1
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(lp, vec, threads, 1)
        if r["value"] is None:
            return {"impl": "reference", "unavailable": r["sample"]}
        if i >= args.warmup:
            vals.append(r)
    v = statistics.median([r["value"] for r in vals])
    secs = statistics.median([r["seconds"] for r in vals])
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(secs * 1e3, 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded lpgen Zipf LP)",
            "config": {"workload": WORKLOAD, "m": lp["m"], "n": lp["n"], "nnz": int(len(lp["ci"]))},
            "cpu_baseline": {"value": v, "unit": "GB/s", "cores": vals[0]["cores"], "kind": "reference",
                             "sample": vals[0]["sample"]},
            "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--only", default="step", choices=["step", "spmv", "spmv_t", "ada", "bb", "gnn", "batch", "price", "gnn_layer",
                             "mps"],
                    help="time one kernel group alone (for profiling); 'step' is the measured workload")
    ap.add_argument("--no-ipm", action="store_true", help="skip the plain GPU IPM solve on the m=2000 LP")
    ap.add_argument("--scale", type=int, default=1, help="--only modes: shrink the LP by this factor (profiling)")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-IPM key")
    ap.add_argument("--no-literal", action="store_true", help="skip the spec-literal (17M nonzeros) SpMV lines")
    ap.add_argument("--no-gnn", action="store_true", help="skip the reduced GNN warm-start key")
    ap.add_argument("--small-gnn", type=int, default=256, help="training and evaluation LPs of the reduced GNN key")
    ap.add_argument("--literal", action="store_true", help="--only spmv / spmv_t: the spec-literal LP")
    ap.add_argument("--spmv-kind", type=int, default=-1, help="--only spmv / spmv_t: pin a path (0 merge, 1 binned)")
    ap.add_argument("--spmv-t", type=int, default=8, help="--only spmv / spmv_t: nonzeros per lane of the binned path")
    ap.add_argument("--ada-layout", type=int, default=-1,
                    help="--only ada: numeric layout (0 gather, 1 row, 2 relative map; -1 the library's choice)")
    ap.add_argument("--batch-k", type=int, default=4096, help="instances in the batched-IPM key")
    ap.add_argument("--batch-sample", type=int, default=4, help="plain GPU IPM solves per size stratum")
    ap.add_argument("--bb-k", type=int, default=2048, help="--only bb: node relaxations")
    ap.add_argument("--bb-chunk", type=int, default=256, help="--only bb: nodes per batched solve")
    ap.add_argument("--gnn-train", type=int, default=1024, help="--only gnn: training LPs")
    ap.add_argument("--gnn-eval", type=int, default=512, help="--only gnn: evaluation LPs")
    ap.add_argument("--gnn-mlo", type=int, default=500, help="--only gnn: smallest m")
    ap.add_argument("--gnn-mhi", type=int, default=5000, help="--only gnn: largest m")
    ap.add_argument("--gnn-epochs", type=int, default=20, help="--only gnn: training epochs")
    ap.add_argument("--gnn-chunk", type=int, default=256, help="--only gnn: LPs per batched solve")
    args = ap.parse_args()
    rank, world, local = dist_setup()
    if args.impl == "reference":
        out = run_reference(args, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    out = run_only(args, local) if args.only != "step" else run_ours(args, rank, world, local)
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
