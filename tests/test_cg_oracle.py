"""The oracle's conjugate-gradient resistance solve M(Y) F = V, pinned against
a dense solve.

The reference declares its operator symmetric positive definite
(src/mobility.jl:161-162) so that Julia Krylov solvers accept it; the oracle's
`cg` restates IterativeSolvers.jl's unpreconditioned iteration and stopping
rule. Here the dense 3N x 3N matrix of the oracle's mobility (one column per
unit force, Float64) gives the exact solution, the symmetry and the
positive-definiteness the iteration relies on.
"""
import math

import numpy as np
import pytest

from fixtures import nonoverlapping_uniform


def _cfg(oracle, N, L, M, T=np.float64):
    return oracle.OracleConfig(T, L=(L, L, L), R_c=3.0, N=N, kernel_widths_ratio=2,
                               num_grid_points=(M, M, M), M_G=8, viscosity=1.0)


@pytest.fixture(scope="module")
def dense_system(oracle):
    N, L, M = 24, 12.0, 16
    cfg = _cfg(oracle, N, L, M)
    Y = nonoverlapping_uniform(N, (L, L, L), seed=11, batch=16)
    cols = []
    for j in range(3 * N):
        e = np.zeros(3 * N)
        e[j] = 1.0
        cols.append(oracle.apply(cfg, Y, e.reshape(N, 3)).reshape(-1))
    Mmat = np.stack(cols, axis=1)
    return cfg, Y, Mmat


def test_mobility_matrix_is_symmetric_positive_definite(dense_system):
    _, _, Mmat = dense_system
    asym = np.abs(Mmat - Mmat.T).max() / np.abs(Mmat).max()
    assert asym < 1e-12
    ev = np.linalg.eigvalsh(0.5 * (Mmat + Mmat.T))
    assert ev.min() > 0


def test_cg_matches_dense_solve_f64(oracle, dense_system):
    cfg, Y, Mmat = dense_system
    N = cfg.N
    V = np.random.default_rng(4).standard_normal((N, 3))
    F, it, res, status = oracle.cg(cfg, Y, V, reltol=1e-12)
    assert status == "converged"
    assert 0 < it <= 3 * N
    exact = np.linalg.solve(Mmat, V.reshape(-1)).reshape(N, 3)
    assert np.linalg.norm(F - exact) / np.linalg.norm(exact) < 1e-9
    # the recursion's residual is the true one to round-off
    true_res = np.linalg.norm(V.reshape(-1) - Mmat @ F.reshape(-1))
    assert abs(true_res - res) <= 1e-10 * np.linalg.norm(V)
    assert res <= 1e-12 * np.linalg.norm(V)


def test_cg_one_iteration_is_the_steepest_descent_step(oracle, dense_system):
    cfg, Y, Mmat = dense_system
    V = np.random.default_rng(5).standard_normal((cfg.N, 3))
    F, it, res, status = oracle.cg(cfg, Y, V, reltol=1e-12, maxiter=1)
    assert (it, status) == (1, "maxiter")
    b = V.reshape(-1)
    alpha = (b @ b) / (b @ (Mmat @ b))
    assert np.allclose(F.reshape(-1), alpha * b, rtol=1e-12, atol=0)
    assert math.isclose(res, np.linalg.norm(b - alpha * (Mmat @ b)), rel_tol=1e-10)


def test_cg_zero_rhs_and_initial_guess(oracle, dense_system):
    cfg, Y, Mmat = dense_system
    N = cfg.N
    F, it, res, status = oracle.cg(cfg, Y, np.zeros((N, 3)))
    assert (it, res, status) == (0, 0.0, "converged") and not F.any()
    V = np.random.default_rng(6).standard_normal((N, 3))
    exact = np.linalg.solve(Mmat, V.reshape(-1)).reshape(N, 3)
    # an initial guess at the solution: |r0| at round-off, abstol stops at once
    F, it, res, status = oracle.cg(cfg, Y, V, x0=exact, abstol=1e-9 * np.linalg.norm(V))
    assert (it, status) == (0, "converged")
    assert np.array_equal(F, exact)


def test_cg_stopping_rule_is_relative_to_the_initial_residual(oracle, dense_system):
    cfg, Y, Mmat = dense_system
    N = cfg.N
    V = np.random.default_rng(7).standard_normal((N, 3))
    x0 = np.random.default_rng(8).standard_normal((N, 3)) * 1e-3
    r0 = np.linalg.norm(V.reshape(-1) - Mmat @ x0.reshape(-1))
    F, it, res, status = oracle.cg(cfg, Y, V, x0=x0, reltol=1e-6)
    assert status == "converged" and res <= 1e-6 * r0
    # one iteration fewer has not yet met it
    _, _, res_prev, st_prev = oracle.cg(cfg, Y, V, x0=x0, reltol=1e-6, maxiter=it - 1)
    assert st_prev == "maxiter" and res_prev > 1e-6 * r0


def test_cg_float32_reaches_its_default_tolerance(oracle):
    N, L, M = 200, 20.0, 32
    Y = nonoverlapping_uniform(N, (L, L, L), seed=12)
    V = np.random.default_rng(9).standard_normal((N, 3))
    c32 = _cfg(oracle, N, L, M, np.float32)
    c64 = _cfg(oracle, N, L, M)
    F32, it32, res32, st32 = oracle.cg(c32, Y.astype(np.float32), V.astype(np.float32))
    F64, it64, _, st64 = oracle.cg(c64, Y, V, reltol=1e-10)
    assert st32 == "converged" and st64 == "converged"
    assert res32 <= math.sqrt(np.finfo(np.float32).eps) * np.linalg.norm(V)
    assert np.linalg.norm(F32 - F64) / np.linalg.norm(F64) < 2e-3
