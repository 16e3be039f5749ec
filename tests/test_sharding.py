"""Ensemble members split across ranks (batched configs 4 and 5): the partition is balanced,
covers every member exactly once, and is computed identically on every rank. Checked with two
`gloo` ranks on CPU: each rank builds its shard of a config-5 ensemble, and the ranks' shards
and per-member totals are gathered and compared."""
import os

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from PlanktonIndividuals import workloads as W
from PlanktonIndividuals.batch import member_cost, shard_members


def test_partition_balanced_and_complete():
    costs = [5.0, 1.0, 3.0, 3.0, 2.0, 8.0, 1.0]
    parts = shard_members(costs, 3)
    flat = sorted(m for p in parts for m in p)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[m] for m in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert shard_members(costs, 1) == [list(range(len(costs)))]
    assert shard_members([], 2) == [[], []]


def _rank(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    boxes = W.config5(n_max=24)
    mine = shard_members([member_cost(w) for w in boxes], ws)[rank]
    ids = torch.full((24,), -1, dtype=torch.int64)
    ids[:len(mine)] = torch.tensor(mine, dtype=torch.int64)
    gathered = [torch.empty_like(ids) for _ in range(ws)]
    dist.all_gather(gathered, ids)
    total = torch.tensor([float(sum(boxes[m].N[0] for m in mine))], dtype=torch.float64)
    dist.all_reduce(total)
    if rank == 0:
        flat = sorted(int(v) for g in gathered for v in g.tolist() if v >= 0)
        out.put((flat, float(total.item()), float(sum(w.N[0] for w in boxes))))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_cover_every_member_once():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    flat, total, expected = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert flat == list(range(24))
    assert total == expected
