"""Adjoint form on the GPU: the pullback of V = M(Y) F (dJ/dY, dJ/dF) against
the oracle's adjoint (itself pinned by finite differences and reverse-mode AD
in tests/test_adjoint_oracle.py) and against central finite differences of the
GPU forward in Float64 at the adjoint workload's full size (N = 100,000,
L = 161, 256^3, M_G = 8, R_c = 3)."""
import numpy as np
import pytest

import ffcm_oracle as O
from fixtures import nonoverlapping_uniform
from gpu_helpers import rel_l2

pytestmark = pytest.mark.gpu


def _kw(N, L, M):
    return dict(L=(L, L, L), R_c=3.0, N=N, kernel_widths_ratio=2.0, viscosity=1.0,
                num_grid_points=(M, M, M), M_G=8)


# (N, L, M): a generic-pipeline case (x length 32 has no register FFT) and the
# fused slab pipeline at the reference's CPU-runnable size
CASES = [(400, 24.0, 32), (2000, 40.0, 64)]


@pytest.mark.parametrize("T", [np.float64, np.float32])
@pytest.mark.parametrize("case", CASES)
def test_pullback_matches_oracle(ffcm, T, case):
    N, L, M = case
    rng = np.random.default_rng(N)
    Y = nonoverlapping_uniform(N, L, seed=N + 1)
    F = rng.standard_normal((N, 3))
    lam = rng.standard_normal((N, 3))
    ora64 = O.OracleConfig(np.float64, **_kw(N, L, M))
    V64, dY64, dF64 = O.adjoint(ora64, Y, F, lam)
    cfg = ffcm.FFCMConfig(T, **_kw(N, L, M))
    Yt, Ft, lt = (a.astype(T) for a in (Y, F, lam))
    V = np.empty((N, 3), T)
    ffcm.mobility_checkpoint(V, cfg, Yt, Ft)
    dY = np.empty((N, 3), T)
    dF = np.empty((N, 3), T)
    ffcm.adjoint(dY, dF, cfg, lt)
    if T == np.float64:
        assert rel_l2(V, V64) < 1e-12
        assert rel_l2(dY, dY64) < 1e-11, rel_l2(dY, dY64)
        assert rel_l2(dF, dF64) < 1e-12, rel_l2(dF, dF64)
    else:
        ora32 = O.OracleConfig(np.float32, **_kw(N, L, M))
        _, dY32, dF32 = O.adjoint(ora32, Yt, Ft, lt)
        e_y, e_f = rel_l2(dY, dY64), rel_l2(dF, dF64)
        print(f"F32 pullback vs F64 oracle: dY {e_y:.2e}, dF {e_f:.2e}; oracle F32 "
              f"{rel_l2(dY32, dY64):.2e}, {rel_l2(dF32, dF64):.2e}")
        assert rel_l2(dF, dF32) < 1e-5
        assert rel_l2(dY, dY32) < 1e-4
        assert e_y < 1e-3 and e_f < 1e-4


def test_pullback_reuses_checkpoint_and_is_linear(ffcm):
    N, L, M = 2000, 40.0, 64
    rng = np.random.default_rng(5)
    Y = nonoverlapping_uniform(N, L, seed=9)
    F = rng.standard_normal((N, 3))
    l1, l2 = rng.standard_normal((N, 3)), rng.standard_normal((N, 3))
    cfg = ffcm.FFCMConfig(np.float64, **_kw(N, L, M))
    V = np.empty((N, 3))
    ffcm.mobility_checkpoint(V, cfg, Y, F)
    out = []
    for lam in (l1, l2, 2.0 * l1 - 3.0 * l2):
        dY, dF = np.empty((N, 3)), np.empty((N, 3))
        ffcm.adjoint(dY, dF, cfg, lam)
        out.append((dY, dF))
    for k in range(2):
        comb = 2.0 * out[0][k] - 3.0 * out[1][k]
        assert rel_l2(out[2][k], comb) < 1e-12


def test_pullback_needs_a_checkpoint(ffcm):
    N, L, M = 400, 24.0, 32
    Y = nonoverlapping_uniform(N, L, seed=1)
    F = np.ones((N, 3))
    cfg = ffcm.FFCMConfig(np.float64, **_kw(N, L, M))
    dY, dF = np.empty((N, 3)), np.empty((N, 3))
    with pytest.raises(ffcm.FFCMError):
        ffcm.adjoint(dY, dF, cfg, F)
    V = np.empty((N, 3))
    ffcm.mobility_checkpoint(V, cfg, Y, F)
    ffcm.adjoint(dY, dF, cfg, F)
    ffcm.mobility(V, cfg, Y, F)          # a plain solve overwrites the checkpoint
    with pytest.raises(ffcm.FFCMError):
        ffcm.adjoint(dY, dF, cfg, F)
    with pytest.raises(ffcm.DimensionMismatch):
        ffcm.adjoint(np.empty((N - 1, 3)), dF, cfg, F)


def test_objective_gradient_host_and_device(ffcm):
    torch = pytest.importorskip("torch")
    N, L, M = 2000, 40.0, 64
    rng = np.random.default_rng(2025)
    Y = nonoverlapping_uniform(N, L, seed=7)
    F = rng.standard_normal((N, 3))
    ora = O.OracleConfig(np.float64, **_kw(N, L, M))
    Vt = O.apply(ora, Y + rng.normal(0, 0.05, Y.shape), F)
    J_o, dY_o, dF_o, V_o = O.objective_gradient(ora, Y, F, Vt)
    cfg = ffcm.FFCMConfig(np.float64, **_kw(N, L, M))
    J, dY, dF, V = ffcm.objective_gradient(cfg, Y, F, Vt)
    assert abs(J - J_o) <= 1e-10 * J_o
    assert rel_l2(V, V_o) < 1e-12 and rel_l2(dY, dY_o) < 1e-11 and rel_l2(dF, dF_o) < 1e-12
    d = lambda a: torch.tensor(a, device="cuda")  # noqa: E731
    Jd, dYd, dFd, Vd = ffcm.objective_gradient(cfg, d(Y), d(F), d(Vt))
    torch.cuda.synchronize()
    assert abs(Jd.item() - J_o) <= 1e-10 * J_o
    assert rel_l2(dYd.cpu().numpy(), dY_o) < 1e-11
    assert rel_l2(dFd.cpu().numpy(), dF_o) < 1e-12


def test_rrule_and_autograd_function(ffcm):
    torch = pytest.importorskip("torch")
    N, L, M = 2000, 40.0, 64
    rng = np.random.default_rng(8)
    Y = nonoverlapping_uniform(N, L, seed=3)
    F = rng.standard_normal((N, 3))
    Vbar = rng.standard_normal((N, 3))
    cfg = ffcm.FFCMConfig(np.float64, **_kw(N, L, M))
    V, pullback = ffcm.rrule_mobility(cfg, Y, F)
    Ybar, Fbar = pullback(Vbar)
    ora = O.OracleConfig(np.float64, **_kw(N, L, M))
    _, dY_o, dF_o = O.adjoint(ora, Y, F, Vbar)
    assert rel_l2(Ybar, dY_o) < 1e-11 and rel_l2(Fbar, dF_o) < 1e-12
    Yt = torch.tensor(Y, device="cuda", requires_grad=True)
    Ft = torch.tensor(F, device="cuda", requires_grad=True)
    Vt = ffcm.mobility_autograd(cfg, Yt, Ft)
    (Vt * torch.tensor(Vbar, device="cuda")).sum().backward()
    assert rel_l2(Yt.grad.cpu().numpy(), dY_o) < 1e-11
    assert rel_l2(Ft.grad.cpu().numpy(), dF_o) < 1e-12


def _far_from_jumps(h, Rc, L, Y, n, i, eps):
    frac = (Y[n, i] / h) % 1.0
    if abs(frac - 0.5) < 4 * eps / h:
        return False
    d = Y - Y[n]
    d -= L * np.round(d / L)
    r = np.sqrt(np.sum(d * d, axis=1))
    r[n] = np.inf
    return bool(np.all(np.abs(r - Rc) > 4 * eps))


def test_gradient_central_differences_full_size(ffcm):
    """J = 0.5 |V(Y, F) - V_t|^2 at N = 100,000, L = 161, 256^3: dJ/dY and dJ/dF
    against central differences (step 1e-4, Float64) at 32 random coordinates;
    the Float32 gradient's error against the Float64 one is printed."""
    torch = pytest.importorskip("torch")
    N, L, M = 100_000, 161.0, 256
    rng = np.random.default_rng(4)
    Y = nonoverlapping_uniform(N, L, seed=44)
    F = rng.standard_normal((N, 3))
    cfg = ffcm.FFCMConfig(np.float64, **_kw(N, L, M))
    dev = lambda a: torch.tensor(np.ascontiguousarray(a), device="cuda")  # noqa: E731
    Yd, Fd = dev(Y), dev(F)
    Vt = torch.empty_like(Yd)
    ffcm.mobility(Vt, cfg, dev(Y + rng.normal(0, 0.05, Y.shape)), Fd)
    J, dY, dF, V64 = ffcm.objective_gradient(cfg, Yd, Fd, Vt)
    lam64 = (V64 - Vt).contiguous()
    dY, dF = dY.cpu().numpy(), dF.cpu().numpy()
    V = torch.empty_like(Yd)

    def Jof(Yp, Fp):
        ffcm.mobility(V, cfg, Yp, Fp)
        return 0.5 * float(((V - Vt) ** 2).sum().item())

    eps, h = 1e-4, float(cfg.h)
    worst_y = worst_f = 0.0
    picked = 0
    while picked < 32:
        n, i = int(rng.integers(N)), int(rng.integers(3))
        if not _far_from_jumps(h, 3.0, L, Y, n, i, eps):
            continue
        picked += 1
        Yp, Ym = Yd.clone(), Yd.clone()
        Yp[n, i] += eps
        Ym[n, i] -= eps
        fd = (Jof(Yp, Fd) - Jof(Ym, Fd)) / (2 * eps)
        Fp, Fm = Fd.clone(), Fd.clone()
        Fp[n, i] += eps
        Fm[n, i] -= eps
        fdF = (Jof(Yd, Fp) - Jof(Yd, Fm)) / (2 * eps)
        scale_y = max(abs(fd), 1e-3 * np.abs(dY).max())
        scale_f = max(abs(fdF), 1e-3 * np.abs(dF).max())
        worst_y = max(worst_y, abs(fd - dY[n, i]) / scale_y)
        worst_f = max(worst_f, abs(fdF - dF[n, i]) / scale_f)
    print(f"central differences at 32 coordinates: worst rel dY {worst_y:.2e}, dF {worst_f:.2e}")
    assert worst_y < 1e-3 and worst_f < 1e-3

    # Float32: the pullback alone (Float64 cotangent rounded to Float32), and
    # end to end, where the residual V - V_t is a small difference of two
    # Float32 solves and carries their rounding (relative 2e-4 of V) amplified
    # by |V| / |V - V_t|
    cfg32 = ffcm.FFCMConfig(np.float32, **_kw(N, L, M))
    Y32, F32 = Yd.float(), Fd.float()
    V32 = torch.empty_like(Y32)
    ffcm.mobility_checkpoint(V32, cfg32, Y32, F32)
    pY, pF = torch.empty_like(Y32), torch.empty_like(Y32)
    ffcm.adjoint(pY, pF, cfg32, lam64.float())
    J32, dY32, dF32, _ = ffcm.objective_gradient(cfg32, Y32, F32, Vt.float())
    torch.cuda.synchronize()
    p_y, p_f = rel_l2(pY.cpu().numpy(), dY), rel_l2(pF.cpu().numpy(), dF)
    e_y = rel_l2(dY32.cpu().numpy(), dY)
    e_f = rel_l2(dF32.cpu().numpy(), dF)
    amp = float(V64.norm() / lam64.norm())
    # the oracle's Float32 pullback on the same inputs: the error the
    # reference's Float32 arithmetic itself carries at this box size
    ora32 = O.OracleConfig(np.float32, **_kw(N, L, M))
    _, oY, oF = O.adjoint(ora32, Y.astype(np.float32), F.astype(np.float32),
                          lam64.cpu().numpy().astype(np.float32))
    o_y, o_f = rel_l2(oY, dY), rel_l2(oF, dF)
    print(f"Float32 pullback vs Float64 (same cotangent): dY {p_y:.2e}, dF {p_f:.2e} "
          f"(oracle Float32: {o_y:.2e}, {o_f:.2e}); end to end: dY {e_y:.2e}, dF {e_f:.2e}, "
          f"J {abs(J32.item() - J.item()) / J.item():.2e}; |V| / |V - V_t| = {amp:.1f}")
    assert p_y <= max(1e-3, 1.05 * o_y) and p_f <= max(1e-4, 1.05 * o_f)
    assert e_y < 1e-3 * amp and e_f < 1e-3 * amp
