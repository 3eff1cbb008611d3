"""One system split over ranks by z slabs (ffcm_dist_*), every rank emulated
in this process on cuda:0 with the collectives done as copies between the
ranks' buffers: the velocities equal the single-GPU solve's, and the oracle's,
for 1 to 4 ranks, both precisions and a non-cubic grid."""
import ctypes

import numpy as np
import pytest

import ffcm_oracle as O
from fixtures import random_cloud
from gpu_helpers import kw_of, rel_l2

pytestmark = pytest.mark.gpu


def _solve(ffcm, T, kw, R, Y, F, stencil=None):
    import torch
    cfgs = [ffcm.DistributedConfig(T, rank=r, nranks=R, stencil=stencil, **kw) for r in range(R)]
    Yd = torch.from_numpy(Y).cuda()
    Fd = torch.from_numpy(F).cuda()
    Vs = [torch.full_like(Yd, float("nan")) for _ in range(R)]
    ffcm.distributed_mobility_local(cfgs, Vs, Yd, Fd)
    torch.cuda.synchronize()
    out = [V.cpu().numpy() for V in Vs]
    ranges = [c.ranges for c in cfgs]
    for c in cfgs:
        c.close()
    return out, ranges


def _single(ffcm, T, kw, Y, F, stencil=None):
    cfg = ffcm.FFCMConfig(T, stencil=stencil, **kw)
    V = np.empty_like(Y)
    ffcm.mobility(V, cfg, Y, F)
    cfg.close()
    return V


@pytest.mark.parametrize("T", [np.float32, np.float64])
@pytest.mark.parametrize("L,M,N,R_c,ranks", [
    (40.0, 64, 2000, 3.0, (1, 2, 3)),
    ((40.0, 40.0, 80.0), (64, 64, 128), 4000, 3.0, (2, 3)),
    (80.0, 128, 20000, 3.0, (2, 4)),
])
def test_dist_matches_single_gpu(ffcm, T, L, M, N, R_c, ranks):
    kw = kw_of(L, N, M, R_c=R_c)
    Lv = kw["L"]
    Y, F = random_cloud(T, N, Lv, 0xD157 + N)
    V1 = _single(ffcm, T, kw, Y, F)
    bound = 2e-6 if T == np.float32 else 1e-13
    for R in ranks:
        Vs, ranges = _solve(ffcm, T, kw, R, Y, F)
        assert ranges[0][0] == 0 and ranges[-1][1] == kw["num_grid_points"][2]
        for V in Vs:                                  # every rank holds all N velocities
            assert np.isfinite(V).all()
            assert rel_l2(V, V1) < bound, (R, rel_l2(V, V1))
        for V in Vs[1:]:
            assert np.array_equal(V, Vs[0])


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_dist_matches_oracle(ffcm, T):
    kw = kw_of(40.0, 2000, 64, R_c=3.0)
    Y, F = random_cloud(T, 2000, kw["L"], 0xD158)
    ora = O.OracleConfig(T, **kw)
    Vo = O.apply(ora, Y, F)
    Vs, _ = _solve(ffcm, T, kw, 3, Y, F)
    assert rel_l2(Vs[0], Vo) < (2e-6 if T == np.float32 else 1e-12)


def test_dist_float64_stencil_geometry(ffcm):
    T = np.float32
    kw = kw_of(40.0, 3000, 64, R_c=3.0)
    Y, F = random_cloud(T, 3000, kw["L"], 0xD159)
    V1 = _single(ffcm, T, kw, Y, F, stencil="float64")
    Vs, _ = _solve(ffcm, T, kw, 2, Y, F, stencil="float64")
    assert rel_l2(Vs[1], V1) < 2e-6


def test_dist_host_arrays(ffcm):
    """Host Y, F and V through the same entry points (the copies inside)."""
    import torch
    T = np.float32
    kw = kw_of(40.0, 2000, 64, R_c=3.0)
    Y, F = random_cloud(T, 2000, kw["L"], 0xD15A)
    V1 = _single(ffcm, T, kw, Y, F)
    cfgs = [ffcm.DistributedConfig(T, rank=r, nranks=2, **kw) for r in range(2)]
    Vs = [np.full_like(Y, np.nan) for _ in range(2)]
    ffcm.distributed_mobility_local(cfgs, Vs, Y, F)
    torch.cuda.synchronize()
    for V in Vs:
        assert rel_l2(V, V1) < 2e-6
    for c in cfgs:
        c.close()


def test_dist_rejects_whole_system_calls_and_bad_grids(ffcm):
    lib = ffcm._lib.load()
    kw = kw_of(40.0, 100, 64, R_c=3.0)
    c = ffcm.DistributedConfig(np.float32, rank=0, nranks=2, **kw)
    Y = np.zeros((100, 3), np.float32)
    V = np.zeros_like(Y)
    rc = lib.ffcm_mobility(c._h, V.ctypes.data, 3, 100, Y.ctypes.data, 3, 100, Y.ctypes.data, 3, 100,
                           ffcm._lib.HOST, None)
    assert rc != 0 and "z-slab" in ffcm._lib.last_error()
    c.close()
    with pytest.raises(ffcm.FFCMError):
        ffcm.DistributedConfig(np.float32, rank=0, nranks=2, **kw_of(40.0, 100, 48, R_c=3.0))
    with pytest.raises(ffcm.ArgumentError):
        ffcm.DistributedConfig(np.float32, rank=0, nranks=1000, **kw)
    plain = ffcm.FFCMConfig(np.float32, **kw)
    rc = lib.ffcm_dist_stokes(plain.handle, None)
    assert rc != 0 and "z-slab" in ffcm._lib.last_error()
    plain.close()


_NCCL_SCRIPT = r"""
import datetime, os, sys
import numpy as np, torch, torch.distributed as dist
sys.path.insert(0, os.path.join(sys.argv[1], "tests"))
from conftest import load_product
from fixtures import random_cloud
ffcm = load_product()
os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=sys.argv[2])
dev = torch.device("cuda", 0)
torch.cuda.set_device(dev)
dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60), device_id=dev)
kw = dict(L=(40.0,) * 3, R_c=3.0, N=2000, kernel_widths_ratio=2.0, viscosity=1.0, num_grid_points=(64,) * 3, M_G=8)
Y, F = random_cloud(np.float32, 2000, kw["L"], 7)
c = ffcm.DistributedConfig(np.float32, rank=0, nranks=1, **kw)
V = torch.empty(2000, 3, device=dev)
c.mobility(V, torch.from_numpy(Y).cuda(), torch.from_numpy(F).cuda(), ffcm.TorchExchange())
one = ffcm.FFCMConfig(np.float32, **kw)
V1 = np.empty_like(Y)
ffcm.mobility(V1, one, Y, F)
err = float(np.linalg.norm(V.cpu().numpy() - V1) / np.linalg.norm(V1))
c.close(); one.close()
dist.destroy_process_group()
print("REL", err)
"""


def test_dist_through_nccl_process_group(tmp_path):
    """DistributedConfig.mobility with TorchExchange over a one-rank NCCL
    process group (the collectives a multi-GPU run makes, on one GPU)."""
    import socket
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    script = tmp_path / "nccl_one_rank.py"
    script.write_text(_NCCL_SCRIPT)
    r = subprocess.run([sys.executable, str(script), str(root), str(port)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    rel = float(r.stdout.split("REL")[-1])
    assert rel < 2e-6
