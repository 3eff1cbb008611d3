"""Pins the oracle's steps 1-2 (wrap, hash, stable counting sort, gather) and the
cold-path geometry against the reference's own known answers:
test/accuracy/test_wrap_positions.jl, test_assign_cells_kernel.jl,
test_assign_cells.jl, test_sort_particles_by_cell.jl, test_cell_geometry.jl,
test_fcm_grid.jl.
"""
import numpy as np
import pytest

import ffcm_oracle as O
from fixtures import fcm_grid_kwargs


# --- test/accuracy/test_wrap_positions.jl ----------------------------------
def test_wrap_upper_boundary_folds_to_zero():
    L = (4.0, 6.0, 8.0)
    Y = np.array([[4.0, 6.0, 8.0]])
    out = np.empty_like(Y)
    O.wrap_positions(out, Y, L)
    assert (out == 0.0).all() and not np.signbit(out).any()


def test_wrap_in_domain_unchanged_and_idempotent():
    L = (4.0, 6.0, 8.0)
    Y = np.array([[1.5, 2.5, 3.5], [0.0, 5.999, 0.0], [3.999, 0.0, 7.999]])
    out = np.empty_like(Y)
    O.wrap_positions(out, Y, L)
    assert (out == Y).all()
    Y2 = np.array([[-1.3, 0.0, 8.5], [9.7, 7.5, -0.1], [-100.0, 20.0, -8.0]])
    once = np.empty_like(Y2)
    O.wrap_positions(once, Y2, L)
    twice = np.empty_like(Y2)
    O.wrap_positions(twice, once, L)
    assert (once == twice).all()


def test_wrap_integer_period_shifts_and_negative_epsilon():
    L = (4.0, 6.0, 8.0)
    base = np.array([[1.5, 2.5, 3.5]])
    ref = np.empty_like(base)
    O.wrap_positions(ref, base, L)
    for k in ((1, 0, 0), (0, 1, 0), (0, 0, 1), (-2, 3, -5)):
        sh = base + np.array(k) * np.array(L)
        out = np.empty_like(sh)
        O.wrap_positions(out, sh, L)
        np.testing.assert_allclose(out, ref, rtol=1e-8)
    eps = 1e-9
    out = np.empty((1, 3))
    O.wrap_positions(out, np.full((1, 3), -eps), L)
    np.testing.assert_allclose(out[0], np.array(L) - eps, rtol=1e-12)


# --- test/accuracy/test_assign_cells_kernel.jl -----------------------------
@pytest.mark.parametrize("Y,num_cells,expected", [
    ((0.5, 0.5, 0.5), (4, 4, 4), 0),
    ((2.5, 2.5, 2.5), (4, 4, 4), 42),
    ((0.5, 2.5, 5.5), (4, 6, 8), 128),
    ((4.0, 4.0, 4.0), (4, 4, 4), 63),   # upper-edge clamp
])
def test_hash_known_answers(Y, num_cells, expected):
    h = np.zeros(1, np.int32)
    O.assign_cells_kernel(h, np.array([Y]), (1.0, 1.0, 1.0), num_cells)
    assert h[0] == expected


def test_hash_bounds_random_cloud():
    rng = np.random.default_rng(2024)
    L = np.array([4.0, 6.0, 8.0])
    Y = rng.random((1000, 3)) * L
    h = np.zeros(1000, np.int32)
    O.assign_cells_kernel(h, Y, (1.0, 1.0, 1.0), (4, 6, 8))
    assert ((0 <= h) & (h < 4 * 6 * 8)).all()


# --- test/accuracy/test_sort_particles_by_cell.jl --------------------------
def _sort(hashes, total):
    h = np.array(hashes, np.int32)
    oi = np.zeros(len(h), np.int32)
    cs = np.zeros(total, np.int32)
    ce = np.zeros(total, np.int32)
    sc = np.zeros(total, np.int32)
    O.build_cell_list_kernel(oi, cs, ce, sc, h)
    return h, oi, cs, ce


def test_sort_orders_by_cell_and_brackets():
    h, oi, cs, ce = _sort([2, 0, 2, 1], 3)
    assert (np.diff(h[oi - 1]) >= 0).all()
    assert sorted(oi.tolist()) == [1, 2, 3, 4]
    covered = []
    for c in range(3):
        for s in range(cs[c], ce[c] + 1):
            assert h[oi[s - 1] - 1] == c
            covered.append(s)
    assert sorted(covered) == [1, 2, 3, 4]
    # exact permutation of the stable counting sort
    assert oi.tolist() == [2, 4, 1, 3]


def test_sort_empty_cell_range():
    _, _, cs, ce = _sort([0, 2, 0, 2], 3)
    assert ce[1] < cs[1]


def test_sort_is_stable():
    _, oi, cs, ce = _sort([0, 1, 0, 1, 0], 2)
    assert oi[cs[0] - 1:ce[0]].tolist() == [1, 3, 5]
    assert oi[cs[1] - 1:ce[1]].tolist() == [2, 4]


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_gather_under_permutation(T):
    rng = np.random.default_rng(2024)
    Y = rng.random((6, 3)).astype(T)
    F = rng.random((6, 3)).astype(T)
    oi = np.array([4, 1, 6, 2, 5, 3], np.int32)
    Ys = np.zeros_like(Y)
    Fs = np.zeros_like(F)
    O.gather_particles_kernel(Ys, Fs, Y, F, oi)
    assert (Ys == Y[oi - 1]).all() and (Fs == F[oi - 1]).all()


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_wrap_hash_sort_groups_random_cloud(T):
    L = (T(4), T(6), T(8))
    cfg = O.OracleConfig(T, L=L, R_c=T(1), N=1000, **fcm_grid_kwargs(L))
    rng = np.random.default_rng(2024)
    Y = (rng.random((1000, 3)) * np.array(L, np.float64)).astype(T)
    F = rng.random((1000, 3)).astype(T)
    O.wrap_positions(Y, Y.copy(), cfg.L)
    O.assign_cells(cfg, Y)
    O.sort_particles_by_cell(cfg, Y, F)
    assert (np.diff(cfg.cell_hash[cfg.original_index - 1]) >= 0).all()
    total = len(cfg.cell_start)
    covered = 0
    for c in range(total):
        for s in range(cfg.cell_start[c], cfg.cell_end[c] + 1):
            assert cfg.cell_hash[cfg.original_index[s - 1] - 1] == c
            covered += 1
    assert covered == 1000
    assert (cfg.Y_sorted == Y[cfg.original_index - 1]).all()
    assert (cfg.F_sorted == F[cfg.original_index - 1]).all()


# --- test/accuracy/test_cell_geometry.jl / test_fcm_grid.jl ----------------
def test_cell_geometry():
    L = (4.0, 6.0, 8.0)
    cfg = O.OracleConfig(np.float64, L=L, R_c=1.0, N=10, **fcm_grid_kwargs(L))
    assert cfg.num_cells == (4, 6, 8)
    for i in range(3):
        assert cfg.cell_size[i] == pytest.approx(L[i] / cfg.num_cells[i])
        assert cfg.inv_cell_size[i] == pytest.approx(1 / cfg.cell_size[i])
        assert cfg.cell_size[i] >= cfg.R_c
    tiny = O.OracleConfig(np.float64, L=(2.0, 2.0, 2.0), R_c=1.0, N=1,
                          **fcm_grid_kwargs((2.0, 2.0, 2.0)))
    assert tiny.num_cells == (3, 3, 3)


def test_constructor_rejections():
    ok = (4.0, 4.0, 4.0)
    kw = fcm_grid_kwargs(ok)
    bad = [dict(L=ok, R_c=0.0, N=1), dict(L=ok, R_c=-1.0, N=1),
           dict(L=(0.0, 4.0, 4.0), R_c=1.0, N=1), dict(L=ok, R_c=1.0, N=0)]
    for b in bad:
        with pytest.raises(O.ArgumentError):
            O.OracleConfig(np.float64, **b, **kw)
    thin = (4.0, 4.0, 2.0)
    with pytest.raises(O.ArgumentError):
        O.OracleConfig(np.float64, L=thin, R_c=1.5, N=1, **fcm_grid_kwargs(thin))
    O.OracleConfig(np.float64, L=thin, R_c=1.0, N=1, **fcm_grid_kwargs(thin))
    base = dict(L=(4.0, 4.0, 4.0), R_c=1.0, N=1, kernel_widths_ratio=2.0,
                num_grid_points=(8, 8, 8), M_G=8, viscosity=1.0)
    for over in (dict(a=2.0), dict(kernel_widths_ratio=0.5), dict(M_G=1), dict(M_G=9),
                 dict(num_grid_points=(0, 8, 8)), dict(viscosity=0.0), dict(viscosity=-1.0),
                 dict(fft_planning="fast"), dict(fft_threads=0),
                 dict(num_grid_points=(8, 8, 16))):
        with pytest.raises(O.ArgumentError):
            O.OracleConfig(np.float64, **{**base, **over})


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_fcm_grid_invariants(T):
    cfg = O.OracleConfig(T, L=(T(4), T(6), T(8)), R_c=T(1), N=1, kernel_widths_ratio=T(2),
                         num_grid_points=(8, 12, 16), M_G=8, viscosity=T(1))
    assert cfg.sigma == T(1) / np.sqrt(T(np.pi))
    assert cfg.Sigma == T(2) * cfg.sigma
    assert cfg.h == T(4) / T(8) and cfg.inv_h == T(1) / cfg.h
    assert len(cfg.k_x) == 5 and len(cfg.k_y) == 12 and len(cfg.k_z) == 16
    assert cfg.k_x[1] == pytest.approx(2 * np.pi / 4, rel=1e-6)
    assert cfg.k_y[12 // 2 + 1] == pytest.approx(2 * np.pi / 6 * (-(12 // 2) + 1), rel=1e-6)
    assert cfg.k_z[-1] == pytest.approx(-2 * np.pi / 8, rel=1e-6)


def test_neighbor_map_half_shell():
    nm = O.build_neighbor_map((3, 4, 5)).reshape(-1, 13)
    # every unordered neighbouring pair of distinct cells appears exactly once
    pairs = set()
    for c, row in enumerate(nm):
        for n in row:
            key = (min(c, n), max(c, n))
            assert key not in pairs
            pairs.add(key)
    assert len(pairs) == 13 * 3 * 4 * 5
