"""Restatement of the reference's shared test fixtures (test/test_utilities.jl)
plus the seeded input generators used by the parity tests and the bench.

Julia's Xoshiro stream is not reproducible from Python; where the reference
draws random inputs with Xoshiro(2024), these helpers draw the same shapes and
ranges from NumPy's default_rng with a stated seed.
"""
from __future__ import annotations

import numpy as np


def near_zero_atol(T):
    """test/test_utilities.jl:8-9."""
    return 1e-6 if np.dtype(T) == np.float32 else 1e-10


def rtol_of(T):
    """Suite convention (test/README.md): relative sqrt(eps(T))."""
    return float(np.sqrt(np.finfo(T).eps))


def fcm_grid_kwargs(L):
    """test/test_utilities.jl:16-27."""
    T = type(L[0])
    h_target = L[0] / 8
    M = tuple(int(round(float(L[i] / h_target))) for i in range(3))
    return dict(kernel_widths_ratio=T(2), num_grid_points=M, M_G=min(8, min(M)),
                viscosity=T(1))


def standard_kwargs(T, N, L=None, num_grid_points=(16, 16, 16), M_G=8, ratio=2.0, mu=1.0,
                    R_c=1.0):
    """test/test_utilities.jl:35-53 (_standard_test_config keywords)."""
    T = np.dtype(T).type
    L = (T(8), T(8), T(8)) if L is None else tuple(T(x) for x in L)
    return dict(L=L, R_c=T(R_c), N=N, kernel_widths_ratio=T(ratio), viscosity=T(mu),
                num_grid_points=num_grid_points, M_G=M_G, fft_planning="estimate")


def clustered_cloud(T, N):
    """test/test_utilities.jl:93-105: 4x4x4 sub-lattice, spacing 0.25, at (4,4,4)."""
    T = np.dtype(T).type
    Y = np.zeros((N, 3), T)
    F = np.zeros((N, 3), T)
    for n in range(1, N + 1):
        Y[n - 1, 0] = T(4) + T(0.25) * T((n - 1) % 4)
        Y[n - 1, 1] = T(4) + T(0.25) * T((n - 1) // 4 % 4)
        Y[n - 1, 2] = T(4) + T(0.25) * T((n - 1) // 16)
        F[n - 1, 0] = T(0.1) * T(n)
        F[n - 1, 1] = T(-0.2) * T(n)
        F[n - 1, 2] = T(0.3) * T(n)
    return Y, F


def random_cloud(T, N, L, seed):
    """Uniform positions in the box, forces U[-0.5, 0.5] (test/cuda/test_gpu_mobility.jl:19-27)."""
    rng = np.random.default_rng(seed)
    T = np.dtype(T).type
    Y = (rng.random((N, 3)) * np.array(L, np.float64)).astype(T)
    F = (rng.random((N, 3)) - 0.5).astype(T)
    return Y, F


def nonoverlapping_uniform(N, L, seed, min_sep=2.0, batch=None, max_phi=0.3):
    """Uniform i.i.d. positions in the box [0, L)^3 (L a scalar or a 3-tuple),
    rejection-sampled so that no two centres are closer than `min_sep` (2a for
    unit spheres).

    Candidates are drawn in batches; a candidate is kept when it is at least
    `min_sep` from every kept centre and from every other candidate of its batch
    (both members of a conflicting in-batch pair are dropped). Neighbour checks
    use a periodic cell grid of side >= min_sep, so the cost is O(N). Returns
    float64 positions of shape (N, 3) in random (shuffled) order.
    """
    rng = np.random.default_rng(seed)
    L = np.broadcast_to(np.asarray(L, np.float64), (3,)).copy()
    phi = N * np.pi / 6.0 * min_sep ** 3 / float(np.prod(L))
    if phi > max_phi:
        raise ValueError(f"volume fraction {phi:.2f} is beyond what random sequential addition "
                         "reaches in reasonable time (0.3)")
    ncv = np.maximum(np.floor(L / min_sep).astype(np.int64), 3)
    cs = L / ncv
    cap = 8
    grid = -np.ones((ncv[0], ncv[1], ncv[2], cap), np.int64)
    fill = np.zeros((ncv[0], ncv[1], ncv[2]), np.int64)
    pos = np.empty((N, 3), np.float64)
    count = 0
    offs = np.array([(dx, dy, dz) for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1)])
    ms2 = min_sep * min_sep
    stalled = 0
    while count < N:
        if stalled > 200:
            raise RuntimeError(f"placed {count} of {N} spheres; no progress in 200 batches")
        need = N - count
        B = batch or max(1024, int(need * 1.3))
        cand = rng.random((B, 3)) * L
        cc = np.minimum((cand / cs).astype(np.int64), ncv - 1)
        ok = np.ones(B, bool)
        # against kept centres
        cu = max(1, int(fill.max()))
        for o in offs:
            nb = (cc + o) % ncv
            occ = grid[nb[:, 0], nb[:, 1], nb[:, 2], :cu]     # (B, cu)
            valid = occ >= 0
            if not valid.any():
                continue
            p = pos[np.where(valid, occ, 0)]                    # (B, cap, 3)
            d = cand[:, None, :] - p
            d -= L * np.round(d / L)
            r2 = np.einsum("bcj,bcj->bc", d, d)
            ok &= ~np.any(valid & (r2 < ms2), axis=1)
        # within the batch: bucket candidates, compare against neighbours
        idx = np.nonzero(ok)[0]
        if idx.size:
            key = (cc[idx, 0] * ncv[1] + cc[idx, 1]) * ncv[2] + cc[idx, 2]
            order = np.argsort(key, kind="stable")
            idx = idx[order]
            key = key[order]
            bad = np.zeros(B, bool)
            starts = np.searchsorted(key, np.arange(int(np.prod(ncv))))
            ends = np.searchsorted(key, np.arange(int(np.prod(ncv))), side="right")
            for o in offs:
                nb = (cc[idx] + o) % ncv
                nk = (nb[:, 0] * ncv[1] + nb[:, 1]) * ncv[2] + nb[:, 2]
                s0, s1 = starts[nk], ends[nk]
                width = int((s1 - s0).max()) if idx.size else 0
                for t in range(width):
                    j = s0 + t
                    m = j < s1
                    if not m.any():
                        continue
                    a = idx[m]
                    b = idx[j[m]]
                    d = cand[a] - cand[b]
                    d -= L * np.round(d / L)
                    r2 = np.einsum("bj,bj->b", d, d)
                    conflict = (a != b) & (r2 < ms2)
                    bad[a[conflict]] = True
            ok &= ~bad
        acc = np.nonzero(ok)[0][:need]
        if acc.size:
            flat = (cc[acc, 0] * ncv[1] + cc[acc, 1]) * ncv[2] + cc[acc, 2]
            order = np.argsort(flat, kind="stable")
            acc, flat = acc[order], flat[order]
            first = np.searchsorted(flat, flat)             # first index of each cell group
            slot = fill.reshape(-1)[flat] + (np.arange(flat.size) - first)
            keep = slot < cap
            acc, flat, slot = acc[keep], flat[keep], slot[keep]
            ids = count + np.arange(acc.size)
            grid.reshape(-1, cap)[flat, slot] = ids
            np.maximum.at(fill.reshape(-1), flat, slot + 1)
            pos[count:count + acc.size] = cand[acc]
            count += acc.size
        stalled = 0 if acc.size else stalled + 1
    perm = rng.permutation(N)
    return pos[perm]


def clustered_gaussian(N, L, nclusters, seed, log_mean=float(np.log(3.0)), log_sigma=0.5):
    """Positions in Gaussian clusters: centres uniform in the cubic box [0, L)^3,
    per-cluster standard deviation log-normal(log_mean, log_sigma), each
    sphere in a uniformly chosen cluster, wrapped into the box.

    No non-overlap test: at the clustered workload's 31% volume fraction,
    rejection sampling jams the cluster cores after a few batches and the
    result is indistinguishable from a uniform placement, so the spheres of a
    cluster may overlap (the method is defined for any distinct positions).
    """
    rng = np.random.default_rng(seed)
    centres = rng.random((nclusters, 3)) * L
    widths = np.exp(rng.normal(log_mean, log_sigma, nclusters))
    c = rng.integers(nclusters, size=N)
    return (centres[c] + rng.standard_normal((N, 3)) * widths[c, None]) % L


def box_for_volume_fraction(N, phi, a=1.0):
    """Cubic box side giving volume fraction phi for N spheres of radius a."""
    return float((N * 4.0 / 3.0 * np.pi * a ** 3 / phi) ** (1.0 / 3.0))


def batched_systems(nsys=64, Nmin=2000, Nmax=64000, phi=0.1, h0=0.54, Mmin=64, Mmax=256, R_c=3.0,
                    seed=2026):
    """The batched workload's suspensions: N log-uniform in [Nmin, Nmax], a
    cubic box at volume fraction phi, and the grid the power of two nearest
    (in log) to L / h0, clamped to [Mmin, Mmax] (so the spacing stays near h0
    and the grids are 64^3, 128^3 or 256^3)."""
    rng = np.random.default_rng(seed)
    Ns = np.exp(rng.uniform(np.log(Nmin), np.log(Nmax), nsys)).astype(np.int64)
    out = []
    for n in Ns:
        L = box_for_volume_fraction(int(n), phi)
        M = int(2 ** int(np.round(np.log2(L / h0))))
        M = min(Mmax, max(Mmin, M))
        out.append(dict(L=(L, L, L), R_c=R_c, N=int(n), num_grid_points=(M, M, M)))
    return out


def batched_inputs(systems, nrhs, seed):
    """Positions (non-overlapping, uniform) and nrhs N(0, 1) force sets per
    system, float64: ([Y_i], [[F_i^r]])."""
    rng = np.random.default_rng(seed + 1)
    Ys = [nonoverlapping_uniform(s["N"], s["L"][0], seed + 10 + i) for i, s in enumerate(systems)]
    Fs = [[rng.standard_normal((s["N"], 3)) for _ in range(nrhs)] for s in systems]
    return Ys, Fs
