"""Pins the oracle's step 6 and the assembled operator against the reference's
known answers: test/accuracy/test_correct_velocities.jl (including its
independent full-tensor oracle), test_single_sphere_mobility.jl (lattice sum),
test_mobility.jl and test_mobility_properties.jl.
"""
import math

import numpy as np
import pytest
from scipy.special import erf

import ffcm_oracle as O
from fixtures import near_zero_atol, rtol_of, standard_kwargs

TS = [np.float32, np.float64]


# --- independent full-tensor oracle (test_correct_velocities.jl:29-68) ------
def _gauss(r2, s2):
    return (2 * math.pi * s2) ** -1.5 * math.exp(-r2 / (2 * s2))


def _S(x, s, mu):
    r = np.linalg.norm(x); r2 = r * r; s2 = s * s
    e = erf(r / (s * math.sqrt(2))); D = _gauss(r2, s2); xx = np.outer(x, x)
    cI = e / (8 * math.pi * mu * r) * (1 + s2 / r2) - s2 ** 2 / (2 * mu * r2) * D
    cxx = e / (8 * math.pi * mu * r ** 3) * (1 - 3 * s2 / r2) + 3 * s2 ** 2 / (2 * mu * r ** 4) * D
    return cI * np.eye(3) + cxx * xx


def _Q(x, s, mu):
    r = np.linalg.norm(x); r2 = r * r; s2 = s * s
    e = erf(r / (s * math.sqrt(2))); D = _gauss(r2, s2); xx = np.outer(x, x)
    cI = e / (4 * math.pi * mu * r ** 3) - (1 + s2 / r2) * D / mu
    cxx = -3 * e / (4 * math.pi * mu * r ** 5) + (1 + 3 * s2 / r2) / (mu * r2) * D
    return cI * np.eye(3) + cxx * xx


def _Tt(x, s, mu):
    r = np.linalg.norm(x); r2 = r * r; s2 = s * s
    D = _gauss(r2, s2); xx = np.outer(x, x)
    return (2 - r2 / s2) / (mu * s2) * D * np.eye(3) + 1 / (mu * s2 ** 2) * D * xx


def correction_tensor(x, sigma, Sigma, mu):
    x = np.asarray(x, np.float64)
    d = sigma ** 2 - Sigma ** 2
    ss, sS = sigma * math.sqrt(2), Sigma * math.sqrt(2)
    return _S(x, ss, mu) - _S(x, sS, mu) - d * _Q(x, sS, mu) - d ** 2 / 4 * _Tt(x, sS, mu)


def _apply_correction(cfg, Y, F):
    Yc = np.array(Y, cfg.T)
    O.wrap_positions(Yc, Yc.copy(), cfg.L)
    O.assign_cells(cfg, Yc)
    O.sort_particles_by_cell(cfg, Yc, np.array(F, cfg.T))
    V = np.zeros((cfg.N, 3), cfg.T)
    O.correct_velocities(V, cfg)
    return V


@pytest.mark.parametrize("T", TS)
def test_sigma_equals_sigma_zero_correction(T):
    s = T(1) / np.sqrt(T(np.pi))
    for mu in (T(0.5), T(1), T(2.7)):
        assert abs(O.self_correction(s, s, T(1), mu)) <= near_zero_atol(T)
        for r in (T(0.2), T(0.75), T(1.5)):
            A, B = O.correction_scalars(r, s, s, mu)
            assert abs(A) <= near_zero_atol(T) and abs(B) <= near_zero_atol(T)


@pytest.mark.parametrize("T", TS)
def test_correction_scalars_match_full_tensor(T):
    s = T(1) / np.sqrt(T(np.pi))
    dirs = [np.array(v, np.float64) / np.linalg.norm(v) for v in
            ((1, 0, 0), (0, 1, 0), (1, 1, 1), (2, -1, 0.5))]
    for ratio in (T(1.5), T(2.5)):
        for mu in (T(0.7), T(1.6)):
            S = ratio * s
            for r in (T(0.3), T(0.6), T(1.2)):
                for d in dirs:
                    x = (r * d.astype(T)).astype(T)
                    A, B = O.correction_scalars(r, s, S, mu)
                    Mi = A * np.eye(3) + B * np.outer(x, x)
                    Mo = correction_tensor(x.astype(np.float64), float(s), float(S), float(mu))
                    np.testing.assert_allclose(Mi, Mo, rtol=rtol_of(T), atol=near_zero_atol(T))


@pytest.mark.parametrize("T", TS)
def test_self_correction_closed_form(T):
    a = T(1)
    s = a / np.sqrt(T(np.pi))
    for ratio in (T(1.25), T(2), T(3.5)):
        for mu in (T(0.5), T(1), T(2.7)):
            S = ratio * s
            Ssp = S * np.sqrt(T(np.pi))
            d = s ** 2 - S ** 2
            ref = (1 / (6 * np.pi * mu * a) - 1 / (6 * np.pi * mu * Ssp)
                   + d / (12 * mu * Ssp ** 3) - d ** 2 / (32 * mu * S ** 5 * np.pi ** 1.5))
            assert O.self_correction(s, S, a, mu) == pytest.approx(float(ref), rel=rtol_of(T))


@pytest.mark.parametrize("T", TS)
def test_isolated_and_two_particle(T):
    cfg = O.OracleConfig(T, **standard_kwargs(T, 2))
    c = O.self_correction(cfg.sigma, cfg.Sigma, cfg.a, cfg.mu)
    F = np.array([[0.3, -0.7, 1.1], [-0.5, 0.9, 0.2]], T)
    V = _apply_correction(cfg, [[1, 1, 1], [4, 4, 4]], F)
    np.testing.assert_allclose(V, c * F, rtol=rtol_of(T), atol=near_zero_atol(T))
    Y = np.array([[4, 4, 4], [4.5, 4.2, 3.8]], T)
    V = _apply_correction(cfg, Y, F)
    x = (Y[0] - Y[1]).astype(np.float64)
    assert np.linalg.norm(x) < cfg.R_c
    M = correction_tensor(x, float(cfg.sigma), float(cfg.Sigma), float(cfg.mu))
    np.testing.assert_allclose(V[0], c * F[0] + M @ F[1], rtol=rtol_of(T), atol=near_zero_atol(T))
    np.testing.assert_allclose(V[1], c * F[1] + M @ F[0], rtol=rtol_of(T), atol=near_zero_atol(T))


@pytest.mark.parametrize("T", TS)
def test_correction_symmetry_linearity_invariance_accumulation(T):
    cfg = O.OracleConfig(T, **standard_kwargs(T, 5))
    Y = np.array([[4.0, 4.0, 4.0], [4.4, 3.8, 4.2], [3.7, 4.3, 4.0], [4.2, 4.1, 3.7],
                  [3.9, 3.6, 4.4]], T)
    Fa = np.array([[0.3, -0.7, 1.1], [-0.5, 0.9, 0.2], [0.8, -0.1, -0.6], [-0.2, 0.5, 0.3],
                   [0.6, -0.4, 0.7]], T)
    Fb = np.array([[-0.2, 0.5, -0.4], [0.6, -0.3, 0.1], [-0.9, 0.7, 0.3], [0.4, -0.8, 0.6],
                   [0.1, 0.2, -0.5]], T)
    Va = _apply_correction(cfg, Y, Fb)
    Vb = _apply_correction(cfg, Y, Fa)
    assert np.sum(Fa * Va, dtype=np.float64) == pytest.approx(
        np.sum(Fb * Vb, dtype=np.float64), rel=rtol_of(T))
    c4 = O.OracleConfig(T, **standard_kwargs(T, 4))
    Y4, F1, F2 = Y[:4], Fa[:4], Fb[:4]
    al, be = T(1.7), T(-0.8)
    Vc = _apply_correction(c4, Y4, al * F1 + be * F2)
    Vs = al * _apply_correction(c4, Y4, F1) + be * _apply_correction(c4, Y4, F2)
    np.testing.assert_allclose(Vc, Vs, rtol=rtol_of(T), atol=near_zero_atol(T))
    Vr = _apply_correction(c4, Y4, F1)
    Vsh = _apply_correction(c4, Y4 + np.array([1.3, -2.1, 0.7], T), F1)
    np.testing.assert_allclose(Vsh, Vr, rtol=rtol_of(T), atol=near_zero_atol(T))
    Yi = Y4.copy()
    Yi[1, 0] += c4.L[0]
    np.testing.assert_allclose(_apply_correction(c4, Yi, F1), Vr, rtol=rtol_of(T),
                               atol=near_zero_atol(T))
    c2 = O.OracleConfig(T, **standard_kwargs(T, 2))
    Y2 = np.array([[4, 4, 4], [4.5, 4.2, 3.8]], T)
    F = np.array([[0.3, -0.7, 1.1], [-0.5, 0.9, 0.2]], T)
    only = _apply_correction(c2, Y2, F)
    V0 = np.array([[2.0, 0.5, -2.5], [-1.0, 3.0, 1.5]], T)
    V = V0.copy()
    O.correct_velocities(V, c2)
    np.testing.assert_allclose(V, V0 + only, rtol=rtol_of(T), atol=near_zero_atol(T))


# --- end to end: test_single_sphere_mobility.jl ---------------------------
def test_single_sphere_lattice_sum_steps_1_to_5():
    T = np.float64
    cfg = O.OracleConfig(T, L=(8.0, 8.0, 8.0), R_c=1.0, N=1, kernel_widths_ratio=1.0,
                         viscosity=1.0, num_grid_points=(32, 32, 32), M_G=21)
    Y = np.array([[4.0, 4.0, 4.0]])
    F = np.array([[1.0, 0.0, 0.0]])
    O.wrap_positions(Y, Y.copy(), cfg.L)
    O.assign_cells(cfg, Y)
    O.sort_particles_by_cell(cfg, Y, F)
    O.spread_forces(cfg)
    O.stokes_solve(cfg)
    V = np.zeros((1, 3))
    O.interpolate_velocities(V, cfg)
    ref = O.periodic_self_mobility_xx(float(cfg.sigma), 1.0, 8.0)
    assert V[0, 0] == pytest.approx(ref, rel=1e-5)
    assert abs(V[0, 1]) <= 1e-12 and abs(V[0, 2]) <= 1e-12
    assert 0 < V[0, 0] < 1 / (6 * math.pi)


def test_single_sphere_sigma_independent_all_six_steps():
    T = np.float64
    s = 1 / math.sqrt(math.pi)
    ref = O.periodic_self_mobility_xx(s, 1.0, 8.0)
    vs = []
    for ratio in (1.25, 1.5):
        cfg = O.OracleConfig(T, L=(8.0, 8.0, 8.0), R_c=1.0, N=1, kernel_widths_ratio=ratio,
                             viscosity=1.0, num_grid_points=(32, 32, 32), M_G=31)
        Y0 = np.array([[4.0, 4.0, 4.0]])
        V = O.apply(cfg, Y0, np.array([[1.0, 0.0, 0.0]]))
        assert (Y0 == 4.0).all()
        assert V[0, 0] == pytest.approx(ref, rel=1e-4)
        assert abs(V[0, 1]) <= 1e-10 and abs(V[0, 2]) <= 1e-10
        vs.append(V[0, 0])
    assert vs[0] == pytest.approx(vs[1], rel=1e-4)


# --- test_mobility.jl -------------------------------------------------------
@pytest.mark.parametrize("T", TS)
def test_mobility_contracts(T):
    cfg = O.OracleConfig(T, **standard_kwargs(T, 4))
    Y = np.array([[9.3, 4.0, 4.0], [4.1, 4.2, 4.0], [-0.4, 4.0, 4.0], [4.0, 9.9, 4.0]], T)
    F = np.array([[0.5, -0.1, 0.2], [-0.3, 0.4, 0.1], [0.2, 0.0, 0.7], [0.1, 0.3, -0.5]], T)
    Y0, F0 = Y.copy(), F.copy()
    O.mobility(np.zeros((4, 3), T), cfg, Y, F)
    assert (Y == Y0).all() and (F == F0).all()
    for bad in (np.zeros((5, 3), T), np.zeros((4, 2), T)):
        with pytest.raises(O.DimensionMismatch):
            O.mobility(bad, cfg, Y, F)
        with pytest.raises(O.DimensionMismatch):
            O.mobility(np.zeros((4, 3), T), cfg, bad, F)
        with pytest.raises(O.DimensionMismatch):
            O.mobility(np.zeros((4, 3), T), cfg, Y, bad)


@pytest.mark.parametrize("T", TS)
def test_mobility_linear_and_spd(T):
    cfg = O.OracleConfig(T, **standard_kwargs(T, 3))
    Y = np.array([[3.5, 4.0, 4.0], [4.6, 4.2, 4.0], [2.0, 6.0, 4.0]], T)
    F = np.array([[0.5, -0.1, 0.2], [-0.3, 0.4, 0.1], [0.2, 0.0, 0.7]], T)
    G = np.array([[0.1, 0.3, -0.2], [0.2, -0.5, 0.4], [-0.4, 0.6, 0.1]], T)
    a, b = T(1.7), T(-0.9)
    VF, VG = O.apply(cfg, Y, F), O.apply(cfg, Y, G)
    Vc = O.apply(cfg, Y, a * F + b * G)
    np.testing.assert_allclose(Vc, a * VF + b * VG, rtol=rtol_of(T), atol=near_zero_atol(T))
    c2 = O.OracleConfig(T, **standard_kwargs(T, 2))
    Y2 = np.array([[3.8, 4.0, 4.0], [4.5, 4.0, 4.0]], T)
    F2 = np.array([[0.5, -0.1, 0.2], [-0.3, 0.4, 0.6]], T)
    G2 = np.array([[0.1, 0.3, -0.4], [0.7, -0.2, 0.5]], T)
    V1, V2 = O.apply(c2, Y2, F2), O.apply(c2, Y2, G2)
    assert np.sum(G2 * V1, dtype=np.float64) == pytest.approx(
        np.sum(F2 * V2, dtype=np.float64), rel=rtol_of(T))
    assert np.sum(F2 * V1, dtype=np.float64) > 0


@pytest.mark.parametrize("T", TS)
def test_mobility_identities_random_configurations(T):
    """test_mobility_properties.jl: seeded random domains (NumPy seed 2024)."""
    rng = np.random.default_rng(2024)
    r, atol = rtol_of(T), near_zero_atol(T)
    for _ in range(6):
        h = T(0.5)
        M = tuple(int(rng.choice([8, 10, 12, 14, 16])) for _ in range(3))
        L = tuple(T(m) * h for m in M)
        N = int(rng.integers(2, 9))
        cfg = O.OracleConfig(T, L=L, R_c=T(1), N=N,
                             kernel_widths_ratio=T(1) + T(1.5) * T(rng.random()),
                             viscosity=T(0.5) + T(2) * T(rng.random()), num_grid_points=M,
                             M_G=int(rng.integers(6, min(M) + 1)))
        Y = np.array([[(T(3) * T(rng.random()) - T(1)) * L[i] for i in range(3)]
                      for _ in range(N)], T)
        F = (T(2) * rng.random((N, 3)) - 1).astype(T)
        G = (T(2) * rng.random((N, 3)) - 1).astype(T)
        a, b = T(2 * rng.random() - 1), T(2 * rng.random() - 1)
        VF, VG = O.apply(cfg, Y, F), O.apply(cfg, Y, G)
        Vc = O.apply(cfg, Y, a * F + b * G)
        np.testing.assert_allclose(Vc, a * VF + b * VG, rtol=r, atol=atol)
        assert np.sum(G * VF, dtype=np.float64) == pytest.approx(
            np.sum(F * VG, dtype=np.float64), rel=r, abs=atol)
        assert np.sum(F * VF, dtype=np.float64) > 0
