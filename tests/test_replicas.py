"""CPU: replica sharding for N>1 GPUs -- LPT balance, and a world-size-2 gloo run in which each
rank aligns its shard (CPU oracle standing in for the per-rank GPU work) and rank 0 gathers the
results back into the original order, equal to a single-process run."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from anchorwave_b200 import replicas
from anchorwave_b200 import workloads as W


def test_lpt_balances_and_covers():
    rng = np.random.default_rng(0)
    costs = [int(c) for c in rng.integers(1, 10**6, size=301)]
    for world in (1, 2, 3, 8):
        sh = replicas.lpt_shards(costs, world)
        assert sorted(i for s in sh for i in s) == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in sh]
        assert max(loads) - min(loads) <= max(costs)


def _worker(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))
    import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ps = W.batched_full_set(24, seed=5, lmax=400)
    costs = [replicas.predicted_cells(len(a), len(b)) for a, b in zip(ps.queries, ps.targets)]
    shards = replicas.lpt_shards(costs, world)
    ora = oracle.Restatement()
    mine = [ora.ksw_extd2(ps.queries[i].tobytes(), ps.targets[i].tobytes(), oracle.anchorwave_matrix(-4),
                          4, 2, 24, 1).key() for i in shards[rank]]
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    if rank == 0:
        q.put(replicas.merge_in_order(len(ps), shards, gathered))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_shard_and_ordered_merge(restatement):
    import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ps = W.batched_full_set(24, seed=5, lmax=400)
    single = [restatement.ksw_extd2(a.tobytes(), b.tobytes(), oracle.anchorwave_matrix(-4), 4, 2, 24, 1).key()
              for a, b in zip(ps.queries, ps.targets)]
    assert merged == single
