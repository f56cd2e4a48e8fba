"""Sharding a batch of LPs over ranks (one process per GPU).

Instances are independent, so a batch shards with no data-path collective:
each rank solves its own instances with the batched GPU IPM and the only
exchange is the final gather of the per-instance results. Instances are
assigned by LPT greedy (largest estimated cost first, each to the least
loaded rank), the cost being the dense normal-matrix factorisation that
dominates a batched solve (m^3 / 3 per iteration) plus the sparse work.
"""
from __future__ import annotations

import heapq

import numpy as np


def instance_cost(m: int, n: int, nnz: int) -> float:
    return m ** 3 / 3.0 + 12.0 * nnz + 8.0 * (m + n)


def lpt_partition(costs, world: int) -> list[np.ndarray]:
    """Index arrays (ascending) per rank; ties go to the lower rank."""
    costs = np.asarray(costs, dtype=np.float64)
    order = np.argsort(-costs, kind="stable")
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(int(i))
        heapq.heappush(heap, (load + costs[i], r))
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def solve_sharded(lps: list, solve_fn, rank: int, world: int, keys=("status", "objective", "iterations"),
                  **kw) -> dict:
    """Runs solve_fn (e.g. hnb200.lp_solve_batch) on this rank's share and
    returns, on every rank, the per-instance `keys` of the whole batch in the
    original order, plus `parts` (the assignment). With world == 1 nothing is
    exchanged."""
    costs = [instance_cost(int(lp["m"]), int(lp["n"]), len(lp["ci"])) for lp in lps]
    parts = lpt_partition(costs, world)
    mine = parts[rank]
    local = {k: np.zeros(0) for k in keys}
    if mine.size:
        sub = {k: ([v[i] for i in mine] if isinstance(v, list) and len(v) == len(lps) else v) for k, v in kw.items()}
        r = solve_fn([lps[i] for i in mine], **sub)
        local = {k: np.asarray(r[k]) for k in keys}
    if world == 1:
        gathered = [local]
    else:
        import torch.distributed as dist

        gathered = [None] * world
        dist.all_gather_object(gathered, local)
    out = {}
    for k in keys:
        dtype = next((g[k].dtype for g in gathered if g[k].size), np.float64)
        full = np.zeros(len(lps), dtype=dtype)
        for r in range(world):
            if parts[r].size:
                full[parts[r]] = gathered[r][k]
        out[k] = full
    out["parts"] = parts
    return out
