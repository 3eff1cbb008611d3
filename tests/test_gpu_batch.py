"""Batched form: every (system, right-hand side) of a graph-launched batch
equals the plain single-system solve and the oracle."""
import numpy as np
import pytest

import ffcm_oracle as O
from fixtures import nonoverlapping_uniform
from gpu_helpers import kw_of, rel_l2

pytestmark = pytest.mark.gpu


def _systems():
    # slab-path systems (power-of-two x, M_G = 8) and a generic-path one
    return [dict(L=(40.0,) * 3, R_c=3.0, N=2000, num_grid_points=(64, 64, 64)),
            dict(L=(60.0,) * 3, R_c=3.0, N=5000, num_grid_points=(128, 128, 128)),
            dict(L=(27.0,) * 3, R_c=3.0, N=400, num_grid_points=(48, 48, 48)),
            dict(L=(32.0, 16.0, 16.0), R_c=2.0, N=300, num_grid_points=(64, 32, 32))]


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_batch_matches_plain_and_oracle(ffcm, T):
    systems = _systems()
    nrhs = 3
    rng = np.random.default_rng(11)
    Ys = [nonoverlapping_uniform(s["N"], s["L"], 100 + i) for i, s in enumerate(systems)]
    Ys = [y.astype(T) for y in Ys]
    Fs = [[rng.standard_normal((s["N"], 3)).astype(T) for _ in range(nrhs)] for s in systems]
    batch = ffcm.FFCMBatch(T, systems=systems, kernel_widths_ratio=2.0, M_G=8, viscosity=1.0,
                           nrhs=nrhs)
    assert batch.kernels_per_call > 0
    Yf, Ff = batch.pack(Ys, Fs)
    V = np.empty_like(Ff)
    batch.mobility(V, Yf, Ff)
    # graph replays reuse the captured buffers; systems run concurrently, so
    # replays also exercise timing-dependent orderings
    tol = 1e-6 if T == np.float32 else 1e-12
    for _ in range(4):
        V2 = np.empty_like(Ff)
        batch.mobility(V2, Yf, Ff)
        assert rel_l2(V2, V) < tol
    parts = batch.unpack(V)
    for i, s in enumerate(systems):
        kw = dict(L=s["L"], R_c=s["R_c"], N=s["N"], kernel_widths_ratio=2.0, viscosity=1.0,
                  num_grid_points=s["num_grid_points"], M_G=8)
        cfg = ffcm.FFCMConfig(T, **kw)
        ora = O.OracleConfig(T, **kw)
        for r in range(nrhs):
            Vp = np.empty_like(Ys[i])
            ffcm.mobility(Vp, cfg, Ys[i], Fs[i][r])
            assert rel_l2(parts[i][r], Vp) < tol
            Vo = O.apply(ora, Ys[i], Fs[i][r])
            assert rel_l2(parts[i][r], Vo) < (1e-5 if T == np.float32 else 1e-10)


def test_batch_device_arrays(ffcm):
    torch = pytest.importorskip("torch")
    systems = _systems()[:2]
    batch = ffcm.FFCMBatch(np.float32, systems=systems, kernel_widths_ratio=2.0, M_G=8,
                           viscosity=1.0, nrhs=2)
    rng = np.random.default_rng(3)
    Ys = [nonoverlapping_uniform(s["N"], s["L"][0], 7 + i).astype(np.float32)
          for i, s in enumerate(systems)]
    Fs = [[rng.standard_normal((s["N"], 3)).astype(np.float32) for _ in range(2)] for s in systems]
    Yf, Ff = batch.pack(Ys, Fs)
    Vh = np.empty_like(Ff)
    batch.mobility(Vh, Yf, Ff)
    Vd = torch.empty(Ff.shape, dtype=torch.float32, device="cuda")
    batch.mobility(Vd, torch.from_numpy(Yf).cuda(), torch.from_numpy(Ff).cuda())
    torch.cuda.synchronize()
    assert rel_l2(Vd.cpu().numpy(), Vh) < 1e-6


def test_batch_rejects_bad_shapes(ffcm):
    batch = ffcm.FFCMBatch(np.float32, systems=_systems()[:1], kernel_widths_ratio=2.0, M_G=8,
                           viscosity=1.0, nrhs=2)
    Y = np.zeros((2000, 3), np.float32)
    with pytest.raises(ffcm.DimensionMismatch):
        batch.mobility(np.zeros((2000, 3), np.float32), Y, np.zeros((2000, 3), np.float32))
