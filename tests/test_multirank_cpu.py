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


def _small_systems():
    # the batched workload's shape at a size the CPU handles in seconds
    import numpy as np
    rng = np.random.default_rng(5)
    out = []
    for i in range(11):
        n = int(rng.integers(20, 300))
        out.append(dict(L=(10.0 + i,) * 3, R_c=1.0, N=n, num_grid_points=(16, 16, 16)))
    return out


def _stand_in_solve(i, Y, F):
    # a host stand-in for the device solve that depends on the system index,
    # the positions and the forces, so any misplaced block shows up
    return F * (1.0 + i) + Y.mean(axis=0)


def _shard_worker(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import numpy as np
    import bench
    from conftest import load_product
    ffcm = load_product()
    systems = _small_systems()
    nrhs = 3
    rng = np.random.default_rng(9)
    Ys_all = [rng.random((s["N"], 3)) * s["L"][0] for s in systems]
    Fs_all = [[rng.standard_normal((s["N"], 3)) for _ in range(nrhs)] for s in systems]
    owner = bench.shard_systems(systems, world)
    mine = [i for i, o in enumerate(owner) if o == rank]
    # this rank's batch: pack its shard, "solve" the packed layout, unpack
    Ns = [systems[i]["N"] for i in mine]
    Yf, Ff = ffcm.pack_batch(np.float64, [Ys_all[i] for i in mine], [Fs_all[i] for i in mine])
    yoff, fvoff = ffcm.batch_offsets(Ns, nrhs)
    Vf = np.empty_like(Ff)
    for k, i in enumerate(mine):
        y = Yf[yoff[k]: yoff[k] + Ns[k]]
        for r in range(nrhs):
            o = fvoff[k] + r * Ns[k]
            Vf[o: o + Ns[k]] = _stand_in_solve(i, y, Ff[o: o + Ns[k]])
    parts = ffcm.unpack_batch(Vf, Ns, nrhs)
    allres = bench.gather_system_results(mine, [[np.array(v) for v in p] for p in parts], len(systems), dist,
                                         rank)
    if rank == 0:
        want = [[_stand_in_solve(i, Ys_all[i], Fs_all[i][r]) for r in range(nrhs)] for i in range(len(systems))]
        ok = all(np.array_equal(allres[i][r], want[i][r]) for i in range(len(systems)) for r in range(nrhs))
        # the checksum does not depend on how the systems were sharded
        one = bench.gather_system_results(list(range(len(systems))), want, len(systems), None, 0)
        out.put((ok, bench.batched_checksum(allres), bench.batched_checksum(one), sorted(set(owner))))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_batch_pack_solve_gather(world):
    """Each gloo rank packs its shard in the batched layout, solves it with a
    host stand-in, unpacks, and rank 0 reassembles all systems in order: the
    result equals the single-process one, block for block."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    ok, cs_sharded, cs_single, ranks_used = q.get(timeout=180)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert ok
    assert cs_sharded == cs_single
    assert ranks_used == list(range(world))


def test_gpus_flag_without_torchrun_launches_ranks(tmp_path):
    """`bench.py --gpus N` outside torchrun starts N ranks itself instead of
    silently running one; inside a launcher the counts must agree."""
    import subprocess
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2", "--steps", "1"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 2 and "WORLD_SIZE=1" in r.stderr
