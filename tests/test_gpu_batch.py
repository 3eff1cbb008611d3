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


def test_batched_workload_at_full_size(ffcm):
    """The batched workload as benchmarked: 64 suspensions (N log-uniform in
    [2000, 64000], 10% volume fraction, 64^3 / 128^3 / 256^3 grids) with 16
    right-hand sides each, Float32. Every (system, right-hand side) equals the
    plain solve of that system; a stratified sample (the smallest and largest
    system of each grid size, alternating right-hand sides) equals the
    oracle."""
    import torch
    from fixtures import batched_inputs, batched_systems
    systems = batched_systems(seed=2024 + 2)
    nrhs = 16
    Ys, Fs = batched_inputs(systems, nrhs, 2024 + 2)
    Ys = [y.astype(np.float32) for y in Ys]
    Fs = [[f.astype(np.float32) for f in fr] for fr in Fs]
    batch = ffcm.FFCMBatch(np.float32, systems=systems, kernel_widths_ratio=2.0, M_G=8, viscosity=1.0,
                           nrhs=nrhs)
    Yf, Ff = batch.pack(Ys, Fs)
    V = np.empty_like(Ff)
    batch.mobility(V, Yf, Ff)
    parts = batch.unpack(V)
    worst = 0.0
    for i, s in enumerate(systems):
        cfg = ffcm.FFCMConfig(np.float32, L=s["L"], R_c=s["R_c"], N=s["N"], kernel_widths_ratio=2.0,
                              viscosity=1.0, num_grid_points=s["num_grid_points"], M_G=8)
        Yd = torch.from_numpy(Ys[i]).cuda()
        for r in range(nrhs):
            Vp = torch.empty_like(Yd)
            ffcm.mobility(Vp, cfg, Yd, torch.from_numpy(Fs[i][r]).cuda())
            torch.cuda.synchronize()
            e = rel_l2(parts[i][r], Vp.cpu().numpy())
            worst = max(worst, e)
        cfg.close()
    assert worst < 1e-6, worst
    sample = []
    for M in sorted({s["num_grid_points"][0] for s in systems}):
        idx = [i for i, s in enumerate(systems) if s["num_grid_points"][0] == M]
        idx.sort(key=lambda i: systems[i]["N"])
        sample += sorted({idx[0], idx[-1]})
    for k, i in enumerate(sample):
        s = systems[i]
        r = (5 * k) % nrhs
        ora = O.OracleConfig(np.float32, L=s["L"], R_c=s["R_c"], N=s["N"], kernel_widths_ratio=2.0,
                             viscosity=1.0, num_grid_points=s["num_grid_points"], M_G=8)
        ora.fft_threads = 8
        e = rel_l2(parts[i][r], O.apply(ora, Ys[i], Fs[i][r]))
        assert e < 1e-5, (i, r, e)
    batch.close()
