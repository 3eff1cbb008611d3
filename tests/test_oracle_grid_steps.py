"""Pins the oracle's steps 3-5 (spread, Stokes solve, interpolation) against the
reference's known answers: test/accuracy/test_spread_forces.jl,
test_modified_kernel_coefficients.jl, test_stokes_solve.jl,
test_interpolate_velocities.jl.
"""
import math

import numpy as np
import pytest

import ffcm_oracle as O
from fixtures import near_zero_atol, rtol_of

TS = [np.float32, np.float64]


def cfg_of(T, L, M, M_G, ratio=2.0, N=1, mu=1.0):
    T = np.dtype(T).type
    if np.isscalar(M):
        M = (M, M, M)
    return O.OracleConfig(T, L=tuple(T(x) for x in L), R_c=T(1), N=N,
                          kernel_widths_ratio=T(ratio), viscosity=T(mu),
                          num_grid_points=M, M_G=M_G)


def closed_form_modified_kernel(T, M, h, Y, sigma, Sigma):
    """Paper eq. (22) expanded: Δ + (σ²−Σ²)/2 ∇²Δ (test_spread_forces.jl:29-43)."""
    T = np.dtype(T).type
    idx = np.arange(M)
    xg = (idx.astype(T) * h)
    Z, Yy, X = np.meshgrid(xg, xg, xg, indexing="ij")
    r2 = (X - Y[0]) ** 2 + (Yy - Y[1]) ** 2 + (Z - Y[2]) ** 2
    D = (T(2) * T(math.pi) * Sigma ** 2) ** (-T(1.5)) * np.exp(-r2 / (T(2) * Sigma ** 2))
    lap = (r2 / Sigma ** 4 - T(3) / Sigma ** 2) * D
    return D + (sigma ** 2 - Sigma ** 2) / T(2) * lap


@pytest.mark.parametrize("T", TS)
def test_modified_kernel_coefficients(T):
    sigma = T(1) / np.sqrt(T(np.pi))
    Sigma = T(1.5) * sigma
    a0, a2, inv_norm, inv_2S2 = O.modified_kernel_coefficients(sigma, Sigma)
    S2 = Sigma * Sigma
    d = sigma * sigma - S2
    r = rtol_of(T)
    assert a0 == pytest.approx(1 - 3 * d / (2 * S2), rel=r)
    assert a2 == pytest.approx(d / (2 * S2 * S2), rel=r)
    assert inv_norm == pytest.approx(1 / np.sqrt(2 * np.pi * S2), rel=r)
    assert inv_2S2 == pytest.approx(1 / (2 * S2), rel=r)
    a0, a2, _, _ = O.modified_kernel_coefficients(sigma, sigma)
    assert a0 == T(1) and a2 == T(0)


# --- spread --------------------------------------------------------------
def _spread_one(cfg, Y, F):
    cfg.Y_sorted[0] = Y
    cfg.F_sorted[0] = F
    O.spread_forces(cfg)
    return cfg.force_density


@pytest.mark.parametrize("T", TS)
def test_spread_closed_form(T):
    cfg = cfg_of(T, (4, 4, 4), 8, 8)
    f = _spread_one(cfg, (2, 2, 2), (1, 0, 0))
    ref = closed_form_modified_kernel(T, 8, cfg.h, (T(2),) * 3, cfg.sigma, cfg.Sigma)
    np.testing.assert_allclose(f[0], ref, rtol=rtol_of(T))
    assert (f[1] == 0).all() and (f[2] == 0).all()


@pytest.mark.parametrize("T", TS)
def test_spread_anchor_convention(T):
    cfg = cfg_of(T, (8, 8, 8), 16, 4)
    for frac, expected in ((0.3, [15, 16, 1, 2]), (0.7, [16, 1, 2, 3])):
        f = _spread_one(cfg, (T(frac) * cfg.h,) * 3, (1, 0, 0))
        marg = np.abs(f[0]).sum(axis=(0, 1))
        assert sorted((np.nonzero(marg > 0)[0] + 1).tolist()) == sorted(expected)


@pytest.mark.parametrize("T", TS)
def test_spread_conservation_and_first_moment(T):
    L = 16
    cfg = cfg_of(T, (L, L, L), 16, 16, N=27)
    for n in range(1, 28):
        nx, ny, nz = (n - 1) % 3 + 1, (n - 1) // 3 % 3 + 1, (n - 1) // 9 + 1
        cfg.Y_sorted[n - 1] = [T(L) * (T(v) - T(0.5)) / T(3) for v in (nx, ny, nz)]
        cfg.F_sorted[n - 1] = [np.sin(T(n)), np.cos(T(n)), T(n) / T(27) - T(0.5)]
    O.spread_forces(cfg)
    h3 = cfg.h ** 3
    for c in range(3):
        assert cfg.force_density[c].sum(dtype=np.float64) * h3 == pytest.approx(
            cfg.F_sorted[:, c].sum(dtype=np.float64), rel=rtol_of(T))
    cfg1 = cfg_of(T, (L, L, L), 16, 16)
    Yn = (T(8.3), T(7.7), T(8.1))
    f = _spread_one(cfg1, Yn, (1, 0, 0))[0].astype(np.float64) * float(cfg1.h) ** 3
    xg = np.arange(16) * float(cfg1.h)
    cent = (np.einsum("zyx,x->", f, xg), np.einsum("zyx,y->", f, xg), np.einsum("zyx,z->", f, xg))
    for i in range(3):
        assert cent[i] == pytest.approx(float(Yn[i]), rel=rtol_of(T))


@pytest.mark.parametrize("T", TS)
def test_spread_translation_linearity_reflection(T):
    cfg = cfg_of(T, (8, 8, 8), 16, 8)
    Ya = (T(2.4), T(3.7), T(5.2))
    fa = _spread_one(cfg, Ya, (1, 2, -3)).copy()
    fc = _spread_one(cfg, (Ya[0] + cfg.h, Ya[1], Ya[2]), (1, 2, -3)).copy()
    np.testing.assert_allclose(np.roll(fa, 1, axis=3), fc, rtol=rtol_of(T), atol=1e-30)
    # linearity with two particles
    cfg2 = cfg_of(T, (16, 16, 16), 16, 8, N=2)
    cfg2.Y_sorted[:] = [[5, 6, 7], [9, 10, 11]]
    al, be = T(1.7), -T(2.3)

    def sp(F1, F2):
        cfg2.F_sorted[:] = [F1, F2]
        O.spread_forces(cfg2)
        return cfg2.force_density.copy()
    f1 = sp((1, 0, 0), (0, 0, 0))
    f2 = sp((0, 0, 0), (0, 1, 2))
    fcmb = sp((al, 0, 0), (0, be, be * 2))
    np.testing.assert_allclose(fcmb, al * f1 + be * f2, rtol=rtol_of(T), atol=1e-30)
    # reflection symmetry about a grid point, odd M_G
    cfg3 = cfg_of(T, (8, 8, 8), 16, 9)
    f = _spread_one(cfg3, (T(4) * cfg3.h,) * 3, (1, 0, 0))[0]
    for d in range(1, 5):
        lo, hi = 4 - d, 4 + d
        assert f[4, 4, lo] == pytest.approx(f[4, 4, hi], rel=rtol_of(T))
        assert f[4, lo, 4] == pytest.approx(f[4, hi, 4], rel=rtol_of(T))
        assert f[lo, 4, 4] == pytest.approx(f[hi, 4, 4], rel=rtol_of(T))


@pytest.mark.parametrize("T", TS)
def test_spread_sigma_equals_sigma_collapse(T):
    cfg = cfg_of(T, (8, 8, 8), 16, 16, ratio=1.0)
    f = _spread_one(cfg, (4, 4, 4), (1, 0, 0))[0]
    s = cfg.sigma
    xg = np.arange(16).astype(T) * cfg.h
    Z, Yy, X = np.meshgrid(xg, xg, xg, indexing="ij")
    r2 = (X - 4) ** 2 + (Yy - 4) ** 2 + (Z - 4) ** 2
    ref = (T(2) * T(np.pi) * s ** 2) ** (-T(1.5)) * np.exp(-r2 / (T(2) * s ** 2))
    np.testing.assert_allclose(f, ref, rtol=rtol_of(T))


# --- Stokes solve -------------------------------------------------------
def _stokes(cfg, fx, fy, fz):
    cfg.force_density[0], cfg.force_density[1], cfg.force_density[2] = fx, fy, fz
    O.stokes_solve(cfg)
    return cfg.fluid_velocity.copy()


def _ijk(M, T):
    iz, iy, ix = np.meshgrid(*(np.arange(1, m + 1).astype(T) for m in M[::-1]), indexing="ij")
    return ix, iy, iz


@pytest.mark.parametrize("T", TS)
def test_stokes_gauge_zero_mean(T):
    cfg = cfg_of(T, (4, 4, 4), 8, 8)
    ix, iy, iz = _ijk((8, 8, 8), T)
    u = _stokes(cfg, ix + iy * T(0.3) - iz * T(0.5) + 1, np.sin(ix + iy) * 2 + T(0.7),
                np.cos(ix * iz) * T(0.5) + T(0.3))
    for c in range(3):
        assert abs(u[c].sum(dtype=np.float64)) <= math.sqrt(np.finfo(T).eps)


@pytest.mark.parametrize("T", TS)
def test_stokes_divergence_free_per_mode(T):
    cfg = cfg_of(T, (4, 4, 4), 8, 8)
    ix, iy, iz = _ijk((8, 8, 8), T)
    f = np.stack([np.sin(ix * T(0.7)) * T(0.5), np.cos(iy + iz * T(0.4)), ix - iy + iz * T(0.2)])
    fh = np.ascontiguousarray(O.forward_transform(cfg, f.astype(T)))
    O.apply_inverse_stokes_kernel(fh, cfg.k_x, cfg.k_y, cfg.k_z, cfg.mu, T(1) / T(512))
    KZ, KY, KX = np.meshgrid(cfg.k_z, cfg.k_y, cfg.k_x, indexing="ij")
    kdotu = KX * fh[0] + KY * fh[1] + KZ * fh[2]
    nrm = np.sqrt(np.abs(fh[0]) ** 2 + np.abs(fh[1]) ** 2 + np.abs(fh[2]) ** 2)
    assert (np.abs(kdotu) <= rtol_of(T) * np.maximum(nrm, 1)).all()


@pytest.mark.parametrize("T", TS)
def test_stokes_single_mode_analytic(T):
    cfg = cfg_of(T, (4, 4, 4), 8, 8, mu=1.5)
    kx = T(2) * T(np.pi) * T(1) / T(4)
    x = (np.arange(8).astype(T) * cfg.h)
    fy = np.broadcast_to(np.sin(kx * x), (8, 8, 8)).astype(T)
    z = np.zeros((8, 8, 8), T)
    u = _stokes(cfg, z, fy, z)
    scale = T(1) / (cfg.mu * kx * kx)
    atol = rtol_of(T) * scale
    assert (np.abs(u[0]) <= atol).all() and (np.abs(u[2]) <= atol).all()
    np.testing.assert_allclose(u[1], np.broadcast_to(scale * np.sin(kx * x), (8, 8, 8)), atol=atol)


@pytest.mark.parametrize("T", TS)
def test_stokes_linearity_shift_viscosity_zero(T):
    cfg = cfg_of(T, (4, 4, 4), 8, 8)
    ix, iy, iz = _ijk((8, 8, 8), T)
    f1 = [np.sin(ix + iy), np.cos(iz * T(0.5)), ix * T(0.1)]
    f2 = [iy - iz * T(0.3), np.sin(ix * iy * T(0.2)), np.cos(iz + ix * T(0.4))]
    al, be = T(1.7), -T(2.3)
    u1 = _stokes(cfg, *f1)
    u2 = _stokes(cfg, *f2)
    uc = _stokes(cfg, *[al * a + be * b for a, b in zip(f1, f2)])
    r = rtol_of(T)
    np.testing.assert_allclose(uc, al * u1 + be * u2, rtol=r, atol=r)
    base = [np.sin(ix + iy), np.cos(iy * iz * T(0.3)), ix - iy * T(0.4)]
    ua = _stokes(cfg, *base)
    ub = _stokes(cfg, *[np.roll(b, 1, axis=2) for b in base])
    np.testing.assert_allclose(ub, np.roll(ua, 1, axis=3), rtol=r, atol=r * np.abs(ua).max())
    hi = cfg_of(T, (4, 4, 4), 8, 8, mu=2.0)
    fy = np.sin(ix * T(0.3) + iy * T(0.2) + iz * T(0.1))
    z = np.zeros_like(fy)
    ul = _stokes(cfg, z, fy, z)
    uh = _stokes(hi, z, fy, z)
    np.testing.assert_allclose(2 * uh, ul, rtol=r, atol=r)
    u0 = _stokes(cfg, z, z, z)
    assert (u0 == 0).all()


@pytest.mark.parametrize("T", TS)
def test_stokes_reflection_equivariance_odd_grid(T):
    cfg = cfg_of(T, (4, 4, 4), 7, 4)
    ix, iy, iz = _ijk((7, 7, 7), T)
    bx = np.sin(ix + iy * T(0.4))
    by = np.cos(ix * T(0.5) + iz)
    bz = ix * T(0.1) - iy * T(0.2) + iz * T(0.3)
    refl = (7 - np.arange(1, 8) + 2 - 1) % 7   # 0-based image of mod1(M - i + 2, M)
    ua = _stokes(cfg, bx, by, bz)
    ub = _stokes(cfg, -bx[:, :, refl], by[:, :, refl], bz[:, :, refl])
    r = rtol_of(T)
    np.testing.assert_allclose(ub[0], -ua[0][:, :, refl], rtol=r, atol=r)
    np.testing.assert_allclose(ub[1], ua[1][:, :, refl], rtol=r, atol=r)
    np.testing.assert_allclose(ub[2], ua[2][:, :, refl], rtol=r, atol=r)


# --- interpolation --------------------------------------------------------
def _field(cfg, fn):
    M = cfg.num_grid_points
    idx = np.arange(1, np.prod(M) + 1).reshape(M[::-1]).astype(cfg.T)
    for c in range(3):
        cfg.fluid_velocity[c] = fn[c](idx)


@pytest.mark.parametrize("T", TS)
def test_interp_adjoint_identity(T):
    cfg = cfg_of(T, (8, 8, 8), 16, 8, N=3)
    cfg.Y_sorted[:] = [[3.1, 3.2, 3.3], [4.5, 4.6, 4.7], [5.2, 2.7, 5.4]]
    cfg.original_index[:] = [1, 2, 3]
    _field(cfg, [lambda i: np.sin(T(0.3) * i), lambda i: np.cos(T(0.2) * i),
                 lambda i: np.sin(T(0.1) * i + 1)])
    V = np.zeros((3, 3), T)
    O.interpolate_velocities(V, cfg)
    u = cfg.fluid_velocity.copy()
    h3 = cfg.h ** 3
    for n in range(3):
        for c in range(3):
            cfg.F_sorted[:] = 0
            cfg.F_sorted[n, c] = 1
            O.spread_forces(cfg)
            adj = h3 * np.sum(u[c] * cfg.force_density[c], dtype=np.float64)
            assert V[n, c] == pytest.approx(adj, rel=rtol_of(T), abs=near_zero_atol(T))


@pytest.mark.parametrize("T", TS)
def test_interp_original_order_and_closed_form(T):
    cfg = cfg_of(T, (8, 8, 8), 16, 8, N=5)
    Y = np.array([[1, 1, 7], [2, 2, 6], [3, 3, 5], [4, 4, 2], [5, 5, 1]], T)
    F = np.zeros_like(Y)
    O.wrap_positions(Y, Y.copy(), cfg.L)
    O.assign_cells(cfg, Y)
    O.sort_particles_by_cell(cfg, Y, F)
    assert cfg.original_index.tolist() != [1, 2, 3, 4, 5]
    fns = [lambda i: np.sin(T(0.17) * i), lambda i: np.cos(T(0.11) * i + T(0.5)),
           lambda i: np.sin(T(0.23) * i - T(0.3))]
    _field(cfg, fns)
    V = np.zeros((5, 3), T)
    O.interpolate_velocities(V, cfg)
    ref = cfg_of(T, (8, 8, 8), 16, 8)
    ref.original_index[0] = 1
    _field(ref, fns)
    for n in range(5):
        ref.Y_sorted[0] = Y[n]
        Vn = np.zeros((1, 3), T)
        O.interpolate_velocities(Vn, ref)
        np.testing.assert_allclose(V[n], Vn[0], rtol=rtol_of(T), atol=near_zero_atol(T))
    # closed form, whole-grid stencil
    c1 = cfg_of(T, (4, 4, 4), 8, 8)
    c1.Y_sorted[0] = (2, 2, 2)
    c1.original_index[0] = 1
    _field(c1, [lambda i: np.sin(T(0.3) * i), lambda i: np.cos(T(0.2) * i),
                lambda i: T(0.05) * i - 1])
    V1 = np.zeros((1, 3), T)
    O.interpolate_velocities(V1, c1)
    K = closed_form_modified_kernel(T, 8, c1.h, (T(2),) * 3, c1.sigma, c1.Sigma)
    for c in range(3):
        ref_v = np.sum(c1.fluid_velocity[c] * K * c1.h ** 3, dtype=np.float64)
        assert V1[0, c] == pytest.approx(ref_v, rel=rtol_of(T), abs=near_zero_atol(T))


@pytest.mark.parametrize("T", TS)
def test_interp_constant_flow_linearity_translation(T):
    cfg = cfg_of(T, (16, 16, 16), 16, 16, N=4)
    cfg.Y_sorted[:] = [[3.3, 4.1, 8.0], [8, 8, 8], [11.7, 2.9, 13.4], [0.4, 15.6, 7.2]]
    cfg.original_index[:] = [1, 2, 3, 4]
    U = (T(0.7), -T(1.3), T(2.1))
    for c in range(3):
        cfg.fluid_velocity[c] = U[c]
    V = np.zeros((4, 3), T)
    O.interpolate_velocities(V, cfg)
    np.testing.assert_allclose(V, np.tile(U, (4, 1)), rtol=rtol_of(T), atol=near_zero_atol(T))
    c2 = cfg_of(T, (8, 8, 8), 16, 8)
    c2.original_index[0] = 1
    _field(c2, [lambda i: np.sin(T(0.3) * i), lambda i: np.cos(T(0.2) * i),
                lambda i: np.sin(T(0.11) * i + T(0.7))])
    base = c2.fluid_velocity.copy()
    Ya = (T(3.4), T(4.7), T(5.2))
    c2.Y_sorted[0] = Ya
    Va = np.zeros((1, 3), T)
    O.interpolate_velocities(Va, c2)
    c2.fluid_velocity[:] = np.roll(base, 1, axis=3)
    c2.Y_sorted[0] = (Ya[0] + c2.h, Ya[1], Ya[2])
    Vb = np.zeros((1, 3), T)
    O.interpolate_velocities(Vb, c2)
    np.testing.assert_allclose(Va, Vb, rtol=rtol_of(T), atol=near_zero_atol(T))


@pytest.mark.parametrize("T", TS)
def test_assembled_grid_operator_symmetric(T):
    cfg = cfg_of(T, (8, 8, 8), 16, 8, N=4)
    Y = np.array([[2.3, 3.1, 4.7], [5.5, 1.9, 6.2], [3.8, 6.6, 2.4], [6.1, 4.2, 5.0]], T)
    O.wrap_positions(Y, Y.copy(), cfg.L)
    O.assign_cells(cfg, Y)

    def app(F):
        O.sort_particles_by_cell(cfg, Y, F)
        O.spread_forces(cfg)
        O.stokes_solve(cfg)
        V = np.zeros((4, 3), T)
        O.interpolate_velocities(V, cfg)
        return V
    n = np.arange(1, 5)[:, None].astype(T)
    i = np.arange(1, 4)[None, :].astype(T)
    Fa = np.sin(n + i).astype(T)
    Fb = np.cos(2 * n - i).astype(T)
    lhs = np.sum(Fa * app(Fb), dtype=np.float64)
    rhs = np.sum(Fb * app(Fa), dtype=np.float64)
    assert lhs == pytest.approx(rhs, rel=rtol_of(T), abs=near_zero_atol(T))
