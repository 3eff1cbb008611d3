"""The oracle's adjoint of the mobility product, pinned two independent ways:

* central finite differences (step 1e-4, Float64) of the oracle's own forward
  (`mobility`, the restatement of src/mobility.jl:23-45);
* reverse-mode automatic differentiation (torch.autograd, Float64) of a
  second, vectorised restatement of the same forward path at N = 2000 (the
  reference's CPU-runnable case: L = 40, 64^3 grid). The reference ships no
  derivative; a ForwardDiff gradient of its CPU path would be the same check
  in Julia.

Finite-difference coordinates avoid the two places where the forward is
discontinuous: the nearest-anchor jump at half-grid positions
(src/stencil.jl:97, round(Y/h)) and the hard pair cutoff r = R_c
(src/correct_velocities.jl:259).
"""
import math

import numpy as np
import pytest

from fixtures import nonoverlapping_uniform

torch = pytest.importorskip("torch")


def _cfg(oracle, N, L, M, T=np.float64):
    return oracle.OracleConfig(T, L=(L, L, L), R_c=3.0, N=N, kernel_widths_ratio=2,
                               num_grid_points=(M, M, M), M_G=8, viscosity=1.0)


def _safe_coordinate(cfg, Y, n, i, eps):
    """False if a +-eps move of Y[n, i] crosses a stencil anchor switch or a cutoff."""
    h = float(cfg.h)
    frac = (float(Y[n, i]) / h) % 1.0
    if abs(frac - 0.5) < 4 * eps / h:
        return False
    L = float(cfg.L[0])
    d = Y - Y[n]
    d -= L * np.round(d / L)
    r = np.sqrt(np.sum(d * d, axis=1))
    r[n] = np.inf
    return bool(np.all(np.abs(r - float(cfg.R_c)) > 4 * eps))


def test_correction_scalar_derivatives_match_difference_quotients(oracle):
    cfg = _cfg(oracle, 8, 24.0, 32)
    for r in (0.3, 0.9, 1.7, 2.4, 2.95):
        A, B, dA, dB = oracle.correction_scalars_d(r, cfg.sigma, cfg.Sigma, cfg.mu)
        assert (A, B) == oracle.correction_scalars(r, cfg.sigma, cfg.Sigma, cfg.mu)
        e = 1e-6
        Ap, Bp = oracle.correction_scalars(r + e, cfg.sigma, cfg.Sigma, cfg.mu)
        Am, Bm = oracle.correction_scalars(r - e, cfg.sigma, cfg.Sigma, cfg.mu)
        assert abs(dA - (Ap - Am) / (2 * e)) <= 1e-7 * max(1.0, abs(dA))
        assert abs(dB - (Bp - Bm) / (2 * e)) <= 1e-7 * max(1.0, abs(dB))


def test_adjoint_matches_central_differences_f64(oracle):
    N, L, M = 400, 24.0, 32
    rng = np.random.default_rng(3)
    Y = nonoverlapping_uniform(N, L, seed=5)
    F = rng.standard_normal((N, 3))
    lam = rng.standard_normal((N, 3))
    cfg = _cfg(oracle, N, L, M)
    V, dY, dF = oracle.adjoint(cfg, Y, F, lam)
    np.testing.assert_array_equal(V, oracle.apply(cfg, Y, F))

    def phi(Yp, Fp):
        return float(np.sum(lam * oracle.apply(cfg, Yp, Fp)))

    eps = 1e-4
    checked = 0
    while checked < 12:
        n, i = int(rng.integers(N)), int(rng.integers(3))
        if not _safe_coordinate(cfg, Y, n, i, eps):
            continue
        Yp, Ym = Y.copy(), Y.copy()
        Yp[n, i] += eps
        Ym[n, i] -= eps
        fd = (phi(Yp, F) - phi(Ym, F)) / (2 * eps)
        assert abs(fd - dY[n, i]) <= 1e-6 * max(abs(fd), 1e-3), (n, i, fd, dY[n, i])
        Fp, Fm = F.copy(), F.copy()
        Fp[n, i] += eps
        Fm[n, i] -= eps
        fdF = (phi(Y, Fp) - phi(Y, Fm)) / (2 * eps)
        assert abs(fdF - dF[n, i]) <= 1e-7 * max(abs(fdF), 1e-3), (n, i, fdF, dF[n, i])
        checked += 1


def test_adjoint_force_part_is_mobility_of_cotangent(oracle):
    N, L, M = 300, 20.0, 32
    rng = np.random.default_rng(11)
    Y = nonoverlapping_uniform(N, L, seed=2)
    F = rng.standard_normal((N, 3))
    lam = rng.standard_normal((N, 3))
    cfg = _cfg(oracle, N, L, M)
    _, _, dF = oracle.adjoint(cfg, Y, F, lam)
    np.testing.assert_allclose(dF, oracle.apply(cfg, Y, lam), rtol=0, atol=1e-14)


# ---------------------------------------------------------------------------
# Reverse-mode AD of an independent restatement of the forward path
# ---------------------------------------------------------------------------

def _torch_objective(cfg, Y, F, Vt):
    """J = 0.5 |V - Vt|^2 with V the mobility product, written with torch ops
    (stencil of src/stencil.jl:80-112, spread src/spread_forces.jl:73-130,
    Stokes src/stokes_solve.jl:21-110, interpolation src/interpolate.jl:82-136,
    correction src/correct_velocities.jl:21-286)."""
    T = torch.float64
    L = float(cfg.L[0])
    Mx, My, Mz = cfg.num_grid_points
    MG = cfg.M_G
    h = float(cfg.h)
    sigma, Sigma, mu = float(cfg.sigma), float(cfg.Sigma), float(cfg.mu)
    S2 = Sigma * Sigma
    dd = sigma * sigma - S2
    a0 = 1 - 3 * dd / (2 * S2)
    a2 = dd / (2 * S2 * S2)
    inv_norm = 1 / math.sqrt(2 * math.pi * S2)

    Yw = torch.remainder(Y, L)
    j = torch.round(Yw.detach() / h).to(torch.int64)                 # (N, 3)
    k = torch.arange(MG, dtype=torch.int64) - MG // 2
    gi = j[:, :, None] + k[None, None, :]                             # (N, 3, MG)
    x = gi.to(T) * h - Yw[:, :, None]
    g = inv_norm * torch.exp(-x * x / (2 * S2))
    r2 = (x[:, 0, :, None, None] ** 2 + x[:, 1, None, :, None] ** 2 + x[:, 2, None, None, :] ** 2)
    w = (a0 + a2 * r2) * g[:, 0, :, None, None] * g[:, 1, None, :, None] * g[:, 2, None, None, :]
    M = torch.tensor([Mx, My, Mz])
    idx = torch.remainder(gi, M[None, :, None])
    flat = (idx[:, 2, None, None, :] * My + idx[:, 1, None, :, None]) * Mx + idx[:, 0, :, None, None]
    N = Y.shape[0]
    w = w.reshape(N, -1)
    flat = flat.reshape(-1)
    plane = Mx * My * Mz
    f = torch.zeros(3, plane, dtype=T)
    f = f.index_add(1, flat, (w[:, :, None] * F[:, None, :]).reshape(-1, 3).T)
    fh = torch.fft.rfftn(f.reshape(3, Mz, My, Mx), dim=(1, 2, 3))
    kx = torch.tensor(np.asarray(cfg.k_x, np.float64))
    ky = torch.tensor(np.asarray(cfg.k_y, np.float64))
    kz = torch.tensor(np.asarray(cfg.k_z, np.float64))
    K = torch.stack(torch.broadcast_tensors(kx[None, None, :], ky[None, :, None], kz[:, None, None]))
    ksq = (K * K).sum(0)
    inv_k2 = torch.where(ksq > 0, 1 / torch.where(ksq > 0, ksq, 1), 0)
    kf = (K * fh).sum(0)
    uh = (fh - K * (kf * inv_k2)) * (inv_k2 / (mu * plane))
    u = torch.fft.irfftn(uh, s=(Mz, My, Mx), dim=(1, 2, 3), norm="forward").reshape(3, plane)
    V = h ** 3 * (w[:, :, None] * u[:, flat].T.reshape(N, -1, 3)).sum(1)

    # pair correction over all pairs within R_c (min image, ties to even)
    Yd = Yw.detach()
    D = Yd[:, None, :] - Yd[None, :, :]
    D = D - L * torch.round(D / L)
    rr = (D * D).sum(-1)
    rr.fill_diagonal_(float("inf"))
    n_i, m_i = torch.nonzero(rr < float(cfg.R_c) ** 2, as_tuple=True)
    xd = Yw[n_i] - Yw[m_i]
    xd = xd - L * torch.round(xd.detach() / L)
    r = torch.sqrt((xd * xd).sum(-1))
    s2, s4, S4 = sigma * sigma, sigma ** 4, S2 * S2
    d = s2 - S2
    dq = d * d / 4
    erf_diff = torch.special.erf(r / (2 * sigma)) - torch.special.erf(r / (2 * Sigma))
    Ds = (4 * math.pi * s2) ** -1.5 * torch.exp(-r * r / (4 * s2))
    DS = (4 * math.pi * S2) ** -1.5 * torch.exp(-r * r / (4 * S2))
    A = (erf_diff * (1 / (8 * math.pi * mu * r) + s2 / (4 * math.pi * mu * r ** 3))
         - 2 * s4 / (mu * r * r) * Ds
         + (2 * S4 / (mu * r * r) + d / mu * (1 + 2 * S2 / (r * r))
            - dq * (2 - r * r / (2 * S2)) / (2 * mu * S2)) * DS)
    B = (erf_diff * (1 / (8 * math.pi * mu * r ** 3) - 3 * s2 / (4 * math.pi * mu * r ** 5))
         + 6 * s4 / (mu * r ** 4) * Ds
         + (-6 * S4 / (mu * r ** 4) - d / (mu * r * r) * (1 + 6 * S2 / (r * r)) - dq / (4 * mu * S4)) * DS)
    Fm = F[m_i]
    dv = A[:, None] * Fm + (B * (xd * Fm).sum(-1))[:, None] * xd
    a = 1.0
    Ssp = Sigma * math.sqrt(math.pi)
    self_c = (1 / (6 * math.pi * mu * a) - 1 / (6 * math.pi * mu * Ssp) + d / (12 * mu * Ssp ** 3)
              - d * d / (32 * mu * Sigma ** 5 * math.sqrt(math.pi ** 3)))
    V = V + self_c * F
    V = V.index_add(0, n_i, dv)
    return 0.5 * ((V - Vt) ** 2).sum(), V


def test_adjoint_matches_reverse_mode_autodiff_n2000(oracle):
    N, L, M = 2000, 40.0, 64
    rng = np.random.default_rng(2025)
    Y = nonoverlapping_uniform(N, L, seed=7)
    F = rng.standard_normal((N, 3))
    cfg = _cfg(oracle, N, L, M)
    Vt = oracle.apply(cfg, Y + rng.normal(0, 0.05, Y.shape), F)
    J, dY, dF, V = oracle.objective_gradient(cfg, Y, F, Vt)

    Yt = torch.tensor(Y, requires_grad=True)
    Ft = torch.tensor(F, requires_grad=True)
    Jt, Vtorch = _torch_objective(cfg, Yt, Ft, torch.tensor(Vt))
    Jt.backward()
    np.testing.assert_allclose(Vtorch.detach().numpy(), V, rtol=0, atol=1e-12)
    assert abs(Jt.item() - J) <= 1e-10 * J
    gY, gF = Yt.grad.numpy(), Ft.grad.numpy()
    rel = lambda a, b: np.linalg.norm(a - b) / np.linalg.norm(b)  # noqa: E731
    assert rel(dY, gY) < 1e-9, rel(dY, gY)
    assert rel(dF, gF) < 1e-9, rel(dF, gF)
