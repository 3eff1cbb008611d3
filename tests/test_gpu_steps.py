"""Step-isolated parity of every hot-path kernel against the oracle, through the
C ABI, mirroring the reference's CPU<->CUDA parity suite (test/cuda/*.jl): each
step reads inputs written identically into both configurations.

* cell list: wrap, hash, ranges, permutation and gather are bit-exact (the
  reference GPU backend only matches the ranges; this backend reproduces the
  stable CPU order);
* spread / Stokes / interpolation / correction: relative-L2 within 2e-6 (F32)
  and 1e-12 (F64) of the oracle, plus the reference's per-element isapprox
  convention (rtol sqrt(eps), atol 1e-6 / 1e-10) where values are O(1).
"""
import numpy as np
import pytest

import ffcm_oracle as O
from fixtures import nonoverlapping_uniform, random_cloud
from gpu_helpers import both, kw_of, rel_l2, tol

pytestmark = pytest.mark.gpu
TS = [np.float32, np.float64]


# ---- cell list ----------------------------------------------------------
@pytest.mark.parametrize("T", TS)
@pytest.mark.parametrize("case", [
    dict(L=8.0, N=1000, M=16, R_c=1.0, half_x=True),
    dict(L=(4.0, 6.0, 8.0), N=1000, M=(8, 12, 16), R_c=1.0, half_x=False),
    dict(L=40.0, N=2000, M=64, R_c=3.0, half_x=False),
    dict(L=100.0, N=100_000, M=64, R_c=3.0, half_x=False),
])
def test_cell_list_bit_exact(ffcm, T, case):
    kw = kw_of(case["L"], case["N"], case["M"], R_c=case["R_c"])
    prod, ora = both(ffcm, T, **kw)
    rng = np.random.default_rng(0xCE11)
    Lv = np.array(kw["L"])
    Y = rng.random((case["N"], 3)) * Lv
    if case["half_x"]:
        Y[:, 0] *= 0.5            # upper-x cells empty: exercises empty ranges
    # shift some particles by whole periods so the wrap has work to do
    Y += rng.integers(-2, 3, size=Y.shape) * Lv
    Y = Y.astype(T)
    F = (rng.random((case["N"], 3)) - 0.5).astype(T)

    ffcm.wrap_positions(prod, Y)
    O.wrap_positions(ora.Y_wrapped, Y, ora.L)
    assert np.array_equal(prod.Y_wrapped, ora.Y_wrapped)
    ffcm.assign_cells(prod)
    O.assign_cells(ora, ora.Y_wrapped)
    assert np.array_equal(prod.cell_hash, ora.cell_hash)
    ffcm.sort_particles_by_cell(prod, F)
    O.sort_particles_by_cell(ora, ora.Y_wrapped, F)
    assert np.array_equal(prod.cell_start, ora.cell_start)
    assert np.array_equal(prod.cell_end, ora.cell_end)
    assert np.array_equal(prod.original_index, ora.original_index)   # stable order
    assert np.array_equal(prod.Y_sorted, ora.Y_sorted)
    assert np.array_equal(prod.F_sorted, ora.F_sorted)
    if case["half_x"]:
        assert (ora.cell_end < ora.cell_start).any()
    nm = prod.get("NEIGHBOR_MAP")
    assert np.array_equal(nm, O.build_neighbor_map(prod.num_cells))


def test_cell_list_deterministic_and_edge_cases(ffcm):
    T = np.float32
    kw = kw_of(8.0, 5, 16, R_c=1.0)
    prod, ora = both(ffcm, T, **kw)
    # upper boundary, exact zero, negative zero, tiny negative, all in one cell
    Y = np.array([[8.0, 8.0, 8.0], [0.0, 0.0, 0.0], [-0.0, 4.0, 7.9999995],
                  [-1e-7, -1e-7, -1e-7], [3.5, 3.5, 3.5]], T)
    F = np.ones((5, 3), T)
    for _ in range(2):
        ffcm.wrap_positions(prod, Y)
        ffcm.assign_cells(prod)
        ffcm.sort_particles_by_cell(prod, F)
    O.wrap_positions(ora.Y_wrapped, Y, ora.L)
    O.assign_cells(ora, ora.Y_wrapped)
    O.sort_particles_by_cell(ora, ora.Y_wrapped, F)
    assert np.array_equal(prod.Y_wrapped.view(np.uint32), ora.Y_wrapped.view(np.uint32))
    assert np.array_equal(prod.cell_hash, ora.cell_hash)
    assert np.array_equal(prod.original_index, ora.original_index)
    # all particles in one cell keep ascending order
    one = np.tile(np.array([[1.5, 1.5, 1.5]], T), (5, 1))
    ffcm.wrap_positions(prod, one)
    ffcm.assign_cells(prod)
    ffcm.sort_particles_by_cell(prod, F)
    assert prod.original_index.tolist() == [1, 2, 3, 4, 5]


# ---- spread -------------------------------------------------------------
def _sorted_inputs(T, N, L, seed):
    rng = np.random.default_rng(seed)
    Y = (rng.random((N, 3)) * np.array(L)).astype(T)
    F = rng.standard_normal((N, 3)).astype(T)
    return Y, F


@pytest.mark.parametrize("T", TS)
@pytest.mark.parametrize("case", [
    dict(L=8.0, N=64, M=16, MG=8),
    dict(L=4.0, N=3, M=8, MG=8),             # stencil covers the whole grid
    dict(L=8.0, N=50, M=16, MG=9),           # odd M_G
    dict(L=(5.0, 6.0, 7.0), N=40, M=(10, 12, 14), MG=6),   # non power of two
    dict(L=40.0, N=2000, M=64, MG=8),
    dict(L=16.0, N=27, M=16, MG=16),
])
def test_spread_parity(ffcm, T, case):
    kw = kw_of(case["L"], case["N"], case["M"], M_G=case["MG"])
    prod, ora = both(ffcm, T, **kw)
    Y, F = _sorted_inputs(T, case["N"], kw["L"], 11)
    prod.set("Y_SORTED", Y)
    prod.set("F_SORTED", F)
    ora.Y_sorted[:] = Y
    ora.F_sorted[:] = F
    ffcm.spread_forces(prod)
    O.spread_forces(ora)
    got, ref = prod.force_density, ora.force_density
    assert rel_l2(got, ref) < tol(T)
    np.testing.assert_allclose(got, ref, rtol=np.sqrt(np.finfo(T).eps),
                               atol=1e-6 * np.abs(ref).max())
    # spreading twice overwrites (the grid is zeroed by every call)
    ffcm.spread_forces(prod)
    assert rel_l2(prod.force_density, ref) < tol(T)


# ---- Stokes solve -------------------------------------------------------
@pytest.mark.parametrize("T", TS)
@pytest.mark.parametrize("M,L", [
    (8, 4.0), (16, 8.0), (7, 4.0), ((10, 12, 14), (5.0, 6.0, 7.0)), ((9, 15, 21), (3.0, 5.0, 7.0)),
    (64, 40.0), ((32, 64, 16), (16.0, 32.0, 8.0)), (128, 64.0), ((22, 26, 34), (11.0, 13.0, 17.0)),
])
def test_stokes_parity(ffcm, T, M, L):
    kw = kw_of(L, 1, M, M_G=2, R_c=min(np.atleast_1d(L)) / 2)
    prod, ora = both(ffcm, T, **kw)
    rng = np.random.default_rng(5)
    f = rng.standard_normal(ora.force_density.shape).astype(T) + T(0.3)
    prod.set("FORCE_DENSITY", f)
    ora.force_density[:] = f
    ffcm.stokes_solve(prod)
    O.stokes_solve(ora)
    got, ref = prod.fluid_velocity, ora.fluid_velocity
    assert rel_l2(got, ref) < (5e-6 if T == np.float32 else 1e-12)
    # gauge: zero mean velocity
    for c in range(3):
        assert abs(got[c].astype(np.float64).mean()) < 1e-5 * np.abs(ref[c]).max()


@pytest.mark.parametrize("T", TS)
def test_stokes_single_mode_analytic(ffcm, T):
    kw = kw_of(4.0, 1, 8, mu=1.5)
    prod = ffcm.FFCMConfig(T, **kw)
    kx = T(2) * T(np.pi) / T(4)
    x = np.arange(8).astype(T) * prod.h
    f = np.zeros((3, 8, 8, 8), T)
    f[1] = np.sin(kx * x)[None, None, :]
    prod.set("FORCE_DENSITY", f)
    ffcm.stokes_solve(prod)
    u = prod.fluid_velocity
    scale = T(1) / (prod.mu * kx * kx)
    atol = np.sqrt(np.finfo(T).eps) * scale
    assert np.abs(u[0]).max() <= atol and np.abs(u[2]).max() <= atol
    np.testing.assert_allclose(u[1], np.broadcast_to(scale * np.sin(kx * x), (8, 8, 8)), atol=atol)
    # zero forcing gives exactly zero velocity
    prod.set("FORCE_DENSITY", np.zeros_like(f))
    ffcm.stokes_solve(prod)
    assert (prod.fluid_velocity == 0).all()


# ---- interpolation ------------------------------------------------------
@pytest.mark.parametrize("T", TS)
@pytest.mark.parametrize("case", [
    dict(L=8.0, N=64, M=16, MG=8), dict(L=4.0, N=3, M=8, MG=8), dict(L=8.0, N=50, M=16, MG=9),
    dict(L=(5.0, 6.0, 7.0), N=40, M=(10, 12, 14), MG=6), dict(L=40.0, N=2000, M=64, MG=8),
])
def test_interpolate_parity(ffcm, T, case):
    kw = kw_of(case["L"], case["N"], case["M"], M_G=case["MG"])
    prod, ora = both(ffcm, T, **kw)
    rng = np.random.default_rng(3)
    Y, _ = _sorted_inputs(T, case["N"], kw["L"], 4)
    u = rng.standard_normal(ora.fluid_velocity.shape).astype(T)
    perm = (rng.permutation(case["N"]) + 1).astype(np.int32)
    prod.set("Y_SORTED", Y)
    prod.set("FLUID_VELOCITY", u)
    prod.set("ORIGINAL_INDEX", perm)
    ora.Y_sorted[:] = Y
    ora.fluid_velocity[:] = u
    ora.original_index[:] = perm
    Vg = np.full((case["N"], 3), np.nan, T)      # overwritten, whatever it held
    ffcm.interpolate_velocities(Vg, prod)
    Vo = np.zeros((case["N"], 3), T)
    O.interpolate_velocities(Vo, ora)
    assert rel_l2(Vg, Vo) < tol(T)
    np.testing.assert_allclose(Vg, Vo, rtol=np.sqrt(np.finfo(T).eps),
                               atol=1e-6 if T == np.float32 else 1e-10)


# ---- correction ---------------------------------------------------------
@pytest.mark.parametrize("T", TS)
@pytest.mark.parametrize("case", [
    dict(L=8.0, N=64, M=16, R_c=1.0, gen="cluster"),
    dict(L=8.0, N=256, M=16, R_c=1.0, gen="random"),
    dict(L=40.0, N=2000, M=64, R_c=3.0, gen="nonoverlap"),
    dict(L=3.0, N=30, M=8, R_c=1.5, gen="random"),        # 3x3x3 cells, self images
])
def test_correct_parity(ffcm, T, case):
    from fixtures import clustered_cloud
    kw = kw_of(case["L"], case["N"], case["M"], R_c=case["R_c"])
    if case["L"] == 3.0:
        kw["M_G"] = 4
    prod, ora = both(ffcm, T, **kw)
    if case["gen"] == "cluster":
        Y, F = clustered_cloud(T, case["N"])
    elif case["gen"] == "random":
        Y, F = random_cloud(T, case["N"], kw["L"], 9)
    else:
        Y = nonoverlapping_uniform(case["N"], case["L"], 7).astype(T)
        F = np.random.default_rng(8).standard_normal((case["N"], 3)).astype(T)
    # CPU-built cell list mirrored to the device (test/cuda/test_gpu_correct.jl:22-32)
    O.wrap_positions(ora.Y_wrapped, Y, ora.L)
    O.assign_cells(ora, ora.Y_wrapped)
    O.sort_particles_by_cell(ora, ora.Y_wrapped, F)
    for name, attr in (("Y_SORTED", "Y_sorted"), ("F_SORTED", "F_sorted"),
                       ("ORIGINAL_INDEX", "original_index"), ("CELL_START", "cell_start"),
                       ("CELL_END", "cell_end")):
        prod.set(name, getattr(ora, attr))
    V0 = np.random.default_rng(1).standard_normal((case["N"], 3)).astype(T)
    Vg = V0.copy()
    ffcm.correct_velocities(Vg, prod)
    Vo = V0.copy()
    O.correct_velocities(Vo, ora)
    # random clouds put pairs far inside 2a, where the pair scalars are small
    # differences of 1/r^3 and 1/r^5 terms: Float32 round-off grows there
    bound = (1e-4 if case["gen"] == "random" else 1e-5) if T == np.float32 else 1e-12
    assert rel_l2(Vg - V0, Vo - V0) < bound
    np.testing.assert_allclose(Vg, Vo, rtol=np.sqrt(np.finfo(T).eps),
                               atol=1e-6 if T == np.float32 else 1e-10)
