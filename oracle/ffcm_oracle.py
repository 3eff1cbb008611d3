"""CPU oracle for the FFCM mobility hot path -- TEST INFRASTRUCTURE ONLY.

A restatement of the reference Julia package ForceCouplingMethod.jl v0.1.0
(Biofluid-Dynamics-Group/FFCM.jl). The particle loops run in plain C
(`oracle/ffcm_oracle.c`, built into `oracle/_build/libffcm_oracle.so` by
`oracle/Makefile`); this module restates the cold path of `src/config.jl`
and drives the six steps of `src/mobility.jl`.

Third-party arithmetic the reference delegates:
  * FFTW 3 through FFTW.jl 1.10 (`plan_rfft` / `plan_brfft`,
    src/config.jl:416-423, src/stokes_solve.jl:21-42). Restated here with
    pocketfft (scipy.fft), which computes the same unnormalised forward
    real-to-complex DFT and the same unnormalised backward complex-to-real
    DFT (the imaginary parts of the x-axis DC and Nyquist bins are ignored by
    the c2r in both libraries).
  * SpecialFunctions 2.8 `erf` (src/correct_velocities.jl:85): C99 `erf`/`erff`.

Only `tests/`, `__graft_entry__.smoke()` and the CPU-baseline leg of
`bench.py` import this module, as the checker. The product never does.

Layouts: a Julia 3xN matrix is a NumPy (N, 3) C-order array; a Julia
(M_x, M_y, M_z) array is a NumPy (M_z, M_y, M_x) C-order array; index buffers
are 1-based as in Julia.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "_build" / "libffcm_oracle.so"
_lib = None


class ArgumentError(ValueError):
    """Mirror of Julia's ArgumentError raised by the parameter checks (src/config.jl:267-312)."""


class DimensionMismatch(ValueError):
    """Mirror of Julia's DimensionMismatch raised by the shape guard (src/mobility.jl:29-34)."""


def build():
    """Compile the C oracle with its Makefile (gcc, no other dependency)."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        _lib = ctypes.CDLL(str(_LIB_PATH))
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _sfx(T):
    return "_f" if T == np.float32 else "_d"


def _ct(T):
    return ctypes.c_float if T == np.float32 else ctypes.c_double


# ----------------------------------------------------------------------------
# Cold path: src/config.jl
# ----------------------------------------------------------------------------

def _wrap_wavevectors(M, L, T):
    """src/config.jl:233-237  per-axis wavevectors in FFTW wrap-around order."""
    twopi = T(2) * T(math.pi)
    half1 = M // 2 + 1
    out = np.empty(M, dtype=T)
    for j in range(1, M + 1):
        m = T(j - 1) if j <= half1 else T(j - 1 - M)
        out[j - 1] = twopi * m / L
    return out


def validate_config_parameters(T, *, L, R_c, N, a, kernel_widths_ratio, num_grid_points, M_G,
                               viscosity, fft_planning, fft_threads):
    """src/config.jl:267-312  _validate_config_parameters (first violation raises)."""
    if not R_c > 0:
        raise ArgumentError("R_c must be positive")
    if not all(x > 0 for x in L):
        raise ArgumentError("L components must be positive")
    if not R_c <= min(L) / T(2):
        raise ArgumentError("R_c must be at most half the smallest box length")
    if not N > 0:
        raise ArgumentError("N must be positive")
    if not a == T(1):
        raise ArgumentError("non-unit particle radius not yet implemented")
    if not kernel_widths_ratio >= T(1):
        raise ArgumentError("kernel widths ratio must be at least 1")
    if not M_G >= 2:
        raise ArgumentError("M_G must be at least 2")
    if not all(m >= 1 for m in num_grid_points):
        raise ArgumentError("num_grid_points components must each be >= 1")
    if not M_G <= min(num_grid_points):
        raise ArgumentError("M_G must not exceed the grid on any axis")
    if not viscosity > 0:
        raise ArgumentError("viscosity must be positive")
    if fft_planning not in ("estimate", "measure", "patient"):
        raise ArgumentError("fft_planning must be :estimate, :measure, or :patient")
    if not fft_threads >= 1:
        raise ArgumentError("fft_threads must be at least 1")


def derive_scalars(T, *, L, R_c, a, kernel_widths_ratio, num_grid_points):
    """src/config.jl:326-359  _derive_scalars, in the working precision T."""
    num_cells = tuple(max(int(np.floor(L[i] / R_c)), 3) for i in range(3))
    cell_size = tuple(L[i] / T(num_cells[i]) for i in range(3))
    inv_cell_size = tuple(T(1) / cell_size[i] for i in range(3))
    sigma = a / np.sqrt(T(math.pi))
    Sigma = kernel_widths_ratio * sigma
    h_axis = tuple(L[i] / T(num_grid_points[i]) for i in range(3))
    rel_tol = np.sqrt(np.finfo(T).eps).astype(T)
    iso = (abs(h_axis[1] - h_axis[0]) <= rel_tol * h_axis[0]
           and abs(h_axis[2] - h_axis[0]) <= rel_tol * h_axis[0])
    if not iso:
        raise ArgumentError("anisotropic grid spacing not supported")
    h = h_axis[0]
    inv_h = T(1) / h
    Mx, My, Mz = num_grid_points
    twopi = T(2) * T(math.pi)
    k_x = np.array([twopi * T(i - 1) / L[0] for i in range(1, Mx // 2 + 2)], dtype=T)
    k_y = _wrap_wavevectors(My, L[1], T)
    k_z = _wrap_wavevectors(Mz, L[2], T)
    return dict(num_cells=num_cells, cell_size=cell_size, inv_cell_size=inv_cell_size,
                sigma=T(sigma), Sigma=T(Sigma), h=T(h), inv_h=T(inv_h),
                k_x=k_x, k_y=k_y, k_z=k_z)


class OracleConfig:
    """CPU restatement of `FFCMConfig{T}` (src/config.jl:196-215, 466-546).

    Holds the derived scalars and the hot-path buffers in the reference layouts.
    """

    def __init__(self, T, *, L, R_c, N, a=None, kernel_widths_ratio, num_grid_points, M_G,
                 viscosity, fft_planning="measure", fft_threads=1, stencil="reference"):
        T = np.dtype(T).type
        self.T = T
        # stencil geometry: "reference" (the reference's arithmetic in T) or
        # "float64" (not the reference: anchors and offsets from the double
        # spacing of the box as given, the library's FFCM_STENCIL_FLOAT64)
        if stencil not in ("reference", "float64"):
            raise ValueError(f"stencil must be 'reference' or 'float64'; got {stencil!r}")
        self.stencil_hd = float(L[0]) / int(num_grid_points[0]) if stencil == "float64" else 0.0
        L = tuple(T(x) for x in L)
        R_c = T(R_c)
        a = T(1) if a is None else T(a)
        ratio = T(kernel_widths_ratio)
        mu = T(viscosity)
        M = tuple(int(m) for m in num_grid_points)
        validate_config_parameters(T, L=L, R_c=R_c, N=N, a=a, kernel_widths_ratio=ratio,
                                   num_grid_points=M, M_G=M_G, viscosity=mu,
                                   fft_planning=fft_planning, fft_threads=fft_threads)
        d = derive_scalars(T, L=L, R_c=R_c, a=a, kernel_widths_ratio=ratio, num_grid_points=M)
        self.L, self.R_c, self.N, self.a, self.mu = L, R_c, int(N), a, mu
        self.num_grid_points, self.M_G = M, int(M_G)
        self.fft_threads = int(fft_threads)
        for k, v in d.items():
            setattr(self, k, v)
        ncell = int(np.prod(self.num_cells))
        N = self.N
        self.cell_hash = np.zeros(N, np.int32)
        self.original_index = np.zeros(N, np.int32)
        self.cell_start = np.zeros(ncell, np.int32)
        self.cell_end = np.zeros(ncell, np.int32)
        self.counting_sort_scratch = np.zeros(ncell, np.int32)
        self.Y_wrapped = np.zeros((N, 3), T)
        self.Y_sorted = np.zeros((N, 3), T)
        self.F_sorted = np.zeros((N, 3), T)
        Mx, My, Mz = M
        self.force_density = np.zeros((3, Mz, My, Mx), T)
        self.fluid_velocity = np.zeros((3, Mz, My, Mx), T)

    # ---- derived helpers -------------------------------------------------
    @property
    def inv_cell_size_arr(self):
        return np.array(self.inv_cell_size, self.T)

    @property
    def L_arr(self):
        return np.array(self.L, self.T)

    @property
    def M_arr(self):
        return np.array(self.num_grid_points, np.int32)

    @property
    def num_cells_arr(self):
        return np.array(self.num_cells, np.int32)


# ----------------------------------------------------------------------------
# Hot path steps (src/cell_list.jl, src/spread_forces.jl, src/stokes_solve.jl,
# src/interpolate.jl, src/correct_velocities.jl)
# ----------------------------------------------------------------------------

def _as_particles(X, T, N=None):
    X = np.ascontiguousarray(np.asarray(X, dtype=T))
    if X.ndim != 2 or X.shape[1] != 3:
        raise DimensionMismatch("expected an (N, 3) array (a Julia 3xN matrix)")
    if N is not None and X.shape[0] != N:
        raise DimensionMismatch("particle count does not match the config")
    return X


def wrap_positions(dst, src, L):
    """src/cell_list.jl:22-31."""
    T = dst.dtype.type
    src = _as_particles(src, T)
    getattr(lib(), "oracle_wrap_positions" + _sfx(T))(
        _p(dst), _p(src), ctypes.c_int64(src.shape[0]), _p(np.array(L, T)))
    return dst


def assign_cells_kernel(cell_hash, Y, inv_cell_size, num_cells):
    """src/cell_list.jl:222-238."""
    T = np.asarray(Y).dtype.type
    Y = _as_particles(Y, T)
    getattr(lib(), "oracle_assign_cells" + _sfx(T))(
        _p(cell_hash), _p(Y), ctypes.c_int64(Y.shape[0]), _p(np.array(inv_cell_size, T)),
        _p(np.array(num_cells, np.int32)))
    return cell_hash


def assign_cells(cfg, Y):
    """src/cell_list.jl:193-198."""
    return assign_cells_kernel(cfg.cell_hash, _as_particles(Y, cfg.T, cfg.N),
                               cfg.inv_cell_size, cfg.num_cells)


def build_cell_list_kernel(original_index, cell_start, cell_end, scratch, cell_hash):
    """src/cell_list.jl:64-93 (stable counting sort, 1-based outputs)."""
    lib().oracle_build_cell_list(
        _p(original_index), _p(cell_start), _p(cell_end), _p(scratch),
        _p(np.ascontiguousarray(cell_hash, np.int32)), ctypes.c_int64(len(cell_hash)),
        ctypes.c_int64(len(cell_start)))
    return original_index


def gather_particles_kernel(Y_sorted, F_sorted, Y, F, original_index):
    """src/cell_list.jl:159-176."""
    T = Y_sorted.dtype.type
    getattr(lib(), "oracle_gather" + _sfx(T))(
        _p(Y_sorted), _p(F_sorted), _p(_as_particles(Y, T)), _p(_as_particles(F, T)),
        _p(np.ascontiguousarray(original_index, np.int32)), ctypes.c_int64(len(original_index)))
    return Y_sorted


def sort_particles_by_cell(cfg, Y, F):
    """src/cell_list.jl:119-133."""
    build_cell_list_kernel(cfg.original_index, cfg.cell_start, cfg.cell_end,
                           cfg.counting_sort_scratch, cfg.cell_hash)
    gather_particles_kernel(cfg.Y_sorted, cfg.F_sorted, Y, F, cfg.original_index)
    return cfg


def build_neighbor_map(num_cells):
    """src/cell_list.jl:258-289."""
    out = np.zeros(13 * int(np.prod(num_cells)), np.int32)
    lib().oracle_build_neighbor_map(_p(out), _p(np.array(num_cells, np.int32)))
    return out


def modified_kernel_coefficients(sigma, Sigma):
    """src/stencil.jl:22-31 -> (a0, a2, inv_norm, inv_2Sigma^2)."""
    T = np.asarray(sigma).dtype.type
    out = np.zeros(4, T)
    ct = _ct(T)
    getattr(lib(), "oracle_modified_kernel_coefficients" + _sfx(T))(
        ct(sigma), ct(Sigma), _p(out))
    return tuple(T(x) for x in out)


def _geometry(cfg):
    """Select the configuration's stencil geometry in the C oracle."""
    lib().oracle_set_stencil_geometry(ctypes.c_double(getattr(cfg, "stencil_hd", 0.0)))


def spread_forces(cfg):
    """src/spread_forces.jl:17-33 / 73-130: overwrite cfg.force_density."""
    _geometry(cfg)
    T = cfg.T
    ct = _ct(T)
    getattr(lib(), "oracle_spread" + _sfx(T))(
        _p(cfg.force_density), _p(cfg.Y_sorted), _p(cfg.F_sorted), ctypes.c_int64(cfg.N),
        ct(cfg.sigma), ct(cfg.Sigma), ct(cfg.h), ct(cfg.inv_h), _p(cfg.M_arr),
        ctypes.c_int32(cfg.M_G))
    return cfg


def forward_transform(cfg, f):
    """Unnormalised r2c over the three axes, x halved (FFTW `plan_rfft`)."""
    import scipy.fft as sfft
    return sfft.rfftn(f, axes=(-3, -2, -1), norm="backward", workers=cfg.fft_threads)


def inverse_transform(cfg, fh):
    """Unnormalised c2r (FFTW `plan_brfft`)."""
    import scipy.fft as sfft
    Mx, My, Mz = cfg.num_grid_points
    return sfft.irfftn(fh, s=(Mz, My, Mx), axes=(-3, -2, -1), norm="forward",
                       workers=cfg.fft_threads)


def apply_inverse_stokes_kernel(fh, k_x, k_y, k_z, mu, inv_M):
    """src/stokes_solve.jl:70-110, in place on fh of shape (3, Mz, My, Mx//2+1)."""
    T = np.asarray(k_x).dtype.type
    assert fh.flags.c_contiguous and fh.dtype == np.dtype(np.complex64 if T == np.float32 else np.complex128)
    ct = _ct(T)
    getattr(lib(), "oracle_apply_inverse_stokes" + _sfx(T))(
        _p(fh), _p(k_x), _p(k_y), _p(k_z), ctypes.c_int64(len(k_x)), ctypes.c_int64(len(k_y)),
        ctypes.c_int64(len(k_z)), ct(mu), ct(inv_M))
    return fh


def stokes_solve(cfg):
    """src/stokes_solve.jl:21-42: force_density -> fluid_velocity."""
    T = cfg.T
    fh = np.ascontiguousarray(forward_transform(cfg, cfg.force_density))
    Mx, My, Mz = cfg.num_grid_points
    inv_M = T(1) / T(Mx * My * Mz)
    apply_inverse_stokes_kernel(fh, cfg.k_x, cfg.k_y, cfg.k_z, cfg.mu, inv_M)
    cfg.fluid_velocity[...] = inverse_transform(cfg, fh)
    return cfg


def interpolate_velocities(V, cfg):
    """src/interpolate.jl:23-42 / 322-376: V[:, original_index[s]] = h^3 * v."""
    _geometry(cfg)
    T = cfg.T
    ct = _ct(T)
    getattr(lib(), "oracle_interpolate" + _sfx(T))(
        _p(V), _p(cfg.fluid_velocity), _p(cfg.Y_sorted), _p(cfg.original_index),
        ctypes.c_int64(cfg.N), ct(cfg.sigma), ct(cfg.Sigma), ct(cfg.h), ct(cfg.inv_h),
        _p(cfg.M_arr), ctypes.c_int32(cfg.M_G))
    return V


def self_correction(sigma, Sigma, a, mu):
    """src/correct_velocities.jl:21-27."""
    T = np.asarray(sigma).dtype.type
    f = getattr(lib(), "oracle_self_correction" + _sfx(T))
    ct = _ct(T)
    f.restype = ct
    return T(f(ct(sigma), ct(Sigma), ct(a), ct(mu)))


def correction_scalars(r, sigma, Sigma, mu):
    """src/correct_velocities.jl:71-104 -> (A, B)."""
    T = np.asarray(sigma).dtype.type
    ct = _ct(T)
    A, B = ct(), ct()
    getattr(lib(), "oracle_correction_scalars" + _sfx(T))(
        ct(r), ct(sigma), ct(Sigma), ct(mu), ctypes.byref(A), ctypes.byref(B))
    return T(A.value), T(B.value)


def correct_velocities(V, cfg):
    """src/correct_velocities.jl:154-173 / 216-286: V += correction."""
    T = cfg.T
    ct = _ct(T)
    getattr(lib(), "oracle_correct" + _sfx(T))(
        _p(V), _p(cfg.Y_sorted), _p(cfg.F_sorted), _p(cfg.cell_start), _p(cfg.cell_end),
        _p(cfg.original_index), _p(cfg.num_cells_arr), _p(cfg.L_arr), ct(cfg.sigma),
        ct(cfg.Sigma), ct(cfg.a), ct(cfg.mu), ct(cfg.R_c))
    return V


def mobility(V, cfg, Y, F):
    """src/mobility.jl:23-45  mobility!(V, config, Y, F) -> V (Y, F untouched)."""
    T = cfg.T
    for name, X in (("V", V), ("Y", Y), ("F", F)):
        X = np.asarray(X)
        if X.shape != (cfg.N, 3):
            raise DimensionMismatch(f"V, Y, and F must each be 3xN for the config's N = {cfg.N}")
    Y = _as_particles(Y, T, cfg.N)
    F = _as_particles(F, T, cfg.N)
    wrap_positions(cfg.Y_wrapped, Y, cfg.L)
    assign_cells(cfg, cfg.Y_wrapped)
    sort_particles_by_cell(cfg, cfg.Y_wrapped, F)
    spread_forces(cfg)
    stokes_solve(cfg)
    interpolate_velocities(V, cfg)
    correct_velocities(V, cfg)
    return V


def apply(cfg, Y, F):
    """Convenience: allocate V and run `mobility`."""
    V = np.zeros((cfg.N, 3), cfg.T)
    return mobility(V, cfg, Y, F)


# ----------------------------------------------------------------------------
# Adjoint (vector-Jacobian product) of the mobility product. The reference
# ships no derivative; this differentiates the restatement above and is pinned
# in the tests by central finite differences of `mobility` in Float64.
# ----------------------------------------------------------------------------

def correction_scalars_d(r, sigma, Sigma, mu):
    """(A, B, dA/dr, dB/dr) of src/correct_velocities.jl:71-104."""
    T = np.asarray(sigma).dtype.type
    ct = _ct(T)
    A, B, dA, dB = ct(), ct(), ct(), ct()
    getattr(lib(), "oracle_correction_scalars_d" + _sfx(T))(
        ct(r), ct(sigma), ct(Sigma), ct(mu), ctypes.byref(A), ctypes.byref(B), ctypes.byref(dA),
        ctypes.byref(dB))
    return T(A.value), T(B.value), T(dA.value), T(dB.value)


def adjoint(cfg, Y, F, lam):
    """Pullback of V = M(Y) F at cotangent `lam` -> (V, dY, dF).

    dF = M lam (M is symmetric); dY is the grid term h^3 sum_g grad w [lam.u + F.psi]
    (u = L^-1 S F kept from the forward, psi = L^-1 S lam) plus the pair term.
    """
    T = cfg.T
    N = cfg.N
    Y = _as_particles(Y, T, N)
    F = _as_particles(F, T, N)
    lam = _as_particles(lam, T, N)
    ct = _ct(T)
    V = np.zeros((N, 3), T)
    mobility(V, cfg, Y, F)
    u = cfg.fluid_velocity.copy()
    F_sorted = cfg.F_sorted.copy()
    L_sorted = np.ascontiguousarray(lam[cfg.original_index.astype(np.int64) - 1])
    cfg.F_sorted[...] = L_sorted
    spread_forces(cfg)
    stokes_solve(cfg)
    psi = cfg.fluid_velocity
    dF = np.zeros((N, 3), T)
    interpolate_velocities(dF, cfg)
    correct_velocities(dF, cfg)
    cfg.F_sorted[...] = F_sorted
    dY = np.zeros((N, 3), T)
    _geometry(cfg)
    getattr(lib(), "oracle_grad_gather" + _sfx(T))(
        _p(dY), _p(u), _p(psi), _p(cfg.Y_sorted), _p(F_sorted), _p(L_sorted),
        _p(cfg.original_index), ctypes.c_int64(N), ct(cfg.sigma), ct(cfg.Sigma), ct(cfg.h),
        ct(cfg.inv_h), _p(cfg.M_arr), ctypes.c_int32(cfg.M_G))
    getattr(lib(), "oracle_correct_grad" + _sfx(T))(
        _p(dY), _p(cfg.Y_sorted), _p(F_sorted), _p(L_sorted), _p(cfg.cell_start),
        _p(cfg.cell_end), _p(cfg.original_index), _p(cfg.num_cells_arr), _p(cfg.L_arr),
        ct(cfg.sigma), ct(cfg.Sigma), ct(cfg.mu), ct(cfg.R_c))
    cfg.fluid_velocity[...] = u
    return V, dY, dF


def objective_gradient(cfg, Y, F, V_target):
    """J = 0.5 |M(Y) F - V_target|^2 and its gradients -> (J, dJ/dY, dJ/dF, V)."""
    T = cfg.T
    V = apply(cfg, Y, F)
    lam = (V - np.asarray(V_target, T)).astype(T)
    V, dY, dF = adjoint(cfg, Y, F, lam)
    J = 0.5 * float(np.sum(lam.astype(np.float64) ** 2))
    return J, dY, dF, V


# ----------------------------------------------------------------------------
# Resistance problem M(Y) F = V by conjugate gradients. The reference ships no
# solver; it declares FFCMMobility symmetric positive definite
# (src/mobility.jl:161-162) so that Julia Krylov packages accept it. This
# restates the unpreconditioned Hestenes-Stiefel iteration in the order and
# with the stopping rule of IterativeSolvers.jl 0.9's `cg` (third-party):
# stop once |r| <= max(reltol |r0|, abstol) or after maxiter iterations.
# Scalars are double; vectors are kept in T, each update rounded once.
# ----------------------------------------------------------------------------

def cg(cfg, Y, V, *, reltol=None, abstol=0.0, maxiter=None, x0=None):
    """-> (F, iters, |r| of the recursion, status) with status 'converged',
    'maxiter' or 'breakdown'."""
    T = cfg.T
    f64 = np.float64
    if reltol is None:
        reltol = math.sqrt(float(np.finfo(T).eps))
    if maxiter is None:
        maxiter = 3 * cfg.N
    b = np.asarray(V, T)
    if x0 is None:
        x = np.zeros((cfg.N, 3), T)
        r = b.copy()
    else:
        x = np.asarray(x0, T).copy()
        r = (b - apply(cfg, Y, x)).astype(T)
    p = np.zeros_like(x)
    rr = float(np.sum(r.astype(f64) ** 2))
    thresh = max(reltol * math.sqrt(rr), abstol)
    if not math.isfinite(rr):
        return x, 0, math.sqrt(rr), "breakdown"
    if math.sqrt(rr) <= thresh:
        return x, 0, math.sqrt(rr), "converged"
    if maxiter <= 0:
        return x, 0, math.sqrt(rr), "maxiter"
    beta = 0.0
    it = 0
    while True:
        p = (r.astype(f64) + beta * p.astype(f64)).astype(T)
        q = apply(cfg, Y, p)
        pq = float(np.sum(p.astype(f64) * q.astype(f64)))
        if not (pq > 0 and math.isfinite(pq)):
            return x, it, math.sqrt(rr), "breakdown"
        alpha = rr / pq
        x = (x.astype(f64) + alpha * p.astype(f64)).astype(T)
        r = (r.astype(f64) - alpha * q.astype(f64)).astype(T)
        rr_new = float(np.sum(r.astype(f64) ** 2))
        beta = rr_new / rr
        rr = rr_new
        it += 1
        if not math.isfinite(rr):
            return x, it, math.sqrt(rr), "breakdown"
        if math.sqrt(rr) <= thresh:
            return x, it, math.sqrt(rr), "converged"
        if it >= maxiter:
            return x, it, math.sqrt(rr), "maxiter"


# ----------------------------------------------------------------------------
# Closed-form references used by the reference's own tests
# ----------------------------------------------------------------------------

def periodic_self_mobility_xx(sigma, mu, Lx, n_max=15):
    """test/test_utilities.jl:112-123  reciprocal-lattice sum (Float64)."""
    n = np.arange(-n_max, n_max + 1, dtype=np.float64)
    nx, ny, nz = np.meshgrid(n, n, n, indexing="ij")
    kx, ky, kz = (2 * np.pi * a / Lx for a in (nx, ny, nz))
    k2 = kx * kx + ky * ky + kz * kz
    mask = k2 > 0
    s = np.sum(np.exp(-sigma ** 2 * k2[mask]) / (mu * k2[mask]) * (1 - kx[mask] ** 2 / k2[mask]))
    return s / Lx ** 3
