"""Helpers shared by the GPU parity tests: matched product/oracle configs and
error metrics. The oracle is the checker; the product runs on cuda:0."""
from __future__ import annotations

import numpy as np

import ffcm_oracle as O


def both(ffcm, T, **kw):
    """A product config and an oracle config with identical parameters."""
    T = np.dtype(T).type
    prod = ffcm.FFCMConfig(T, **kw)
    ora = O.OracleConfig(T, **kw)
    return prod, ora


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a - b))


def tol(T):
    """Relative-L2 bound for a product-vs-oracle comparison in precision T."""
    return 2e-6 if np.dtype(T) == np.float32 else 1e-12


def kw_of(L, N, M, M_G=8, R_c=1.0, ratio=2.0, mu=1.0):
    if np.isscalar(L):
        L = (L, L, L)
    if np.isscalar(M):
        M = (M, M, M)
    return dict(L=tuple(float(x) for x in L), R_c=R_c, N=N, kernel_widths_ratio=ratio,
                viscosity=mu, num_grid_points=M, M_G=M_G, fft_planning="estimate")
