"""Multi-rank host logic on CPU (gloo, world size 2): the batched form shards
independent systems across ranks with no data-path collective; every system is
owned by exactly one rank, the shards balance the cost model, and the
max-over-ranks timing reduction the bench uses works."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    systems = bench.batched_systems()
    owner = bench.shard_systems(systems, world)
    mine = torch.tensor([i for i, o in enumerate(owner) if o == rank], dtype=torch.int64)
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(sizes, torch.tensor([mine.numel()]))
    gathered = [torch.zeros(int(s.item()), dtype=torch.int64) for s in sizes]
    # all_gather needs equal sizes: pad to the max
    m = max(int(s.item()) for s in sizes)
    padded = torch.full((m,), -1, dtype=torch.int64)
    padded[: mine.numel()] = mine
    allp = [torch.zeros(m, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(allp, padded)
    t = torch.tensor([float(rank + 1)])
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        owned = sorted(int(x) for a in allp for x in a.tolist() if x >= 0)
        out.put((owned, len(systems), float(t.item())))
    dist.barrier()
    dist.destroy_process_group()


def test_batched_sharding_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    owned, n, tmax = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert owned == list(range(n))        # every system exactly once
    assert tmax == 2.0                    # max over ranks


def test_shard_balance():
    sys.path.insert(0, str(ROOT))
    import bench
    import numpy as np
    systems = bench.batched_systems()
    for world in (1, 2, 4, 8):
        owner = bench.shard_systems(systems, world)
        cost = [s["N"] * 512 + 3 * np.prod(s["num_grid_points"]) * np.log2(np.prod(s["num_grid_points"]))
                for s in systems]
        loads = [sum(c for c, o in zip(cost, owner) if o == r) for r in range(world)]
        assert sorted(set(owner)) == list(range(world))
        assert max(loads) <= 1.35 * (sum(loads) / world) + max(cost)
