"""Host logic of the z-slab decomposition of one system over ranks
(ffcm_dist_partition, and the collectives of TorchExchange on gloo ranks):
no GPU work."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.parametrize("T", [np.float32, np.float64])
@pytest.mark.parametrize("M", [(64, 64, 64), (512, 512, 512), (256, 128, 64), (1024, 1024, 1024)])
def test_partition_covers_planes_and_columns(ffcm, T, M):
    nkx = M[0] // 2 + 1
    one = ffcm.dist_partition(T, M, 1, 0)
    assert one == (0, M[2], 0, nkx)
    R = 1
    while True:
        try:
            parts = [ffcm.dist_partition(T, M, R, r) for r in range(R)]
        except ffcm.ArgumentError:
            break
        z = [(a, b) for a, b, _, _ in parts]
        k = [(c, d) for _, _, c, d in parts]
        assert z[0][0] == 0 and z[-1][1] == M[2] and k[0][0] == 0 and k[-1][1] == nkx
        for (a, b), (c, d) in zip(z, z[1:]):
            assert b == c
        for (a, b), (c, d) in zip(k, k[1:]):
            assert b == c
        widths = [b - a for a, b in z]
        assert min(widths) > 0 and min(b - a for a, b in k) > 0
        slab = np.gcd.reduce(widths + [M[2]])
        assert max(widths) - min(widths) <= slab      # balanced to one slab
        R = R * 2 + 1
    assert R > 3, "at least three ranks fit every grid here"


def test_partition_rejects_bad_arguments(ffcm):
    with pytest.raises(ffcm.ArgumentError):
        ffcm.dist_partition(np.float32, (64, 64, 64), 2, 2)
    with pytest.raises(ffcm.ArgumentError):
        ffcm.dist_partition(np.float32, (64, 64, 64), 0, 0)
    with pytest.raises(ffcm.ArgumentError, match="more ranks"):
        ffcm.dist_partition(np.float32, (64, 64, 64), 1000, 0)
    with pytest.raises(ffcm.FFCMError):
        ffcm.dist_partition(np.float32, (96, 64, 64), 2, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, str(ROOT / "tests"))
    from conftest import load_product
    ffcm = load_product()
    ex = ffcm.TorchExchange()
    blk = 6
    # send block q of rank r holds 100 r + q: after the transpose, block q of
    # rank r's receive buffer must hold 100 q + r (what rank q sent to r)
    send = torch.tensor([100 * rank + q for q in range(world) for _ in range(blk)], dtype=torch.float32)
    recv = torch.full_like(send, -1.0)
    ex.all_to_all(recv, send)
    partial = torch.full((9,), float(rank + 1))
    ex.all_reduce(partial)
    out.put((rank, recv.view(world, blk)[:, 0].tolist(), partial[0].item()))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_torch_exchange_routes_blocks(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict((r, (recv, s)) for r, recv, s in (q.get(timeout=180) for _ in range(world)))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        recv, s = got[r]
        assert recv == [100.0 * qq + r for qq in range(world)]
        assert s == world * (world + 1) / 2
