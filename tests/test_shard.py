"""CPU: sharding a batch of LPs over ranks (shard.py) -- the LPT partition,
and the gather of per-instance results through torch.distributed with two
gloo ranks (world_size 2, 127.0.0.1). The GPU solve is replaced by a
deterministic stand-in so the distributed plumbing runs without a GPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import lpgen
import shard


def fake_solve(lps, **kw):
    """Stand-in for hnb200.lp_solve_batch: status 1, objective = sum(c),
    iterations = m (+ the warm-start marker when one is given)."""
    extra = kw.get("x0s")
    return {"status": np.ones(len(lps), np.int32),
            "objective": np.array([float(np.sum(lp["c"])) for lp in lps]),
            "iterations": np.array([lp["m"] + (0 if extra is None else int(extra[i][0])) for i, lp in enumerate(lps)])}


def batch(k=23, seed=0):
    rng = np.random.default_rng(seed)
    return [lpgen.lp_uniform(int(m), int(2.5 * m), 4, 70 + i) for i, m in enumerate(rng.integers(10, 80, k))]


def test_lpt_partition_covers_and_balances():
    rng = np.random.default_rng(1)
    costs = rng.uniform(1, 100, 101) ** 3
    for world in (1, 2, 3, 8):
        parts = shard.lpt_partition(costs, world)
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(101))
        loads = [costs[p].sum() for p in parts]
        # LPT bound: max load <= optimum + largest job <= mean + max
        assert max(loads) <= np.mean(loads) + costs.max() + 1e-9
    assert [p.tolist() for p in shard.lpt_partition([5, 5, 5, 5], 2)] == [[0, 2], [1, 3]]


def test_single_rank_matches_direct_solve():
    lps = batch()
    r = shard.solve_sharded(lps, fake_solve, 0, 1)
    d = fake_solve(lps)
    for k in ("status", "objective", "iterations"):
        assert np.array_equal(r[k], d[k])


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lps = batch()
        x0s = [np.full(lp["n"], float(i % 3)) for i, lp in enumerate(lps)]
        r = shard.solve_sharded(lps, fake_solve, rank, world, x0s=x0s)
        q.put((rank, {k: r[k].tolist() for k in ("status", "objective", "iterations")},
               [p.tolist() for p in r["parts"]]))
    finally:
        dist.destroy_process_group()


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.timeout(120)
def test_two_gloo_ranks_gather_the_whole_batch():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=100) for _ in procs]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    lps = batch()
    x0s = [np.full(lp["n"], float(i % 3)) for i, lp in enumerate(lps)]
    d = fake_solve(lps, x0s=x0s)
    for rank, res, parts in out:
        assert sorted(parts[0] + parts[1]) == list(range(len(lps))) and parts[0] and parts[1]
        for k in ("status", "objective", "iterations"):
            assert np.array_equal(np.array(res[k]), d[k]), (rank, k)
