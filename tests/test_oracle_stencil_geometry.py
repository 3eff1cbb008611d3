"""The oracle's Float64 stencil geometry option (the library's
FFCM_STENCIL_FLOAT64 mode, not part of the reference): particles whose Y / h
lies within Float32 rounding of a half-integer take different stencil anchors
in Float32 and Float64 arithmetic, which dominates the Float32 result's
distance from Float64; anchors and offsets from the double box spacing remove
it. Host only."""
import numpy as np

import ffcm_oracle as O


def _flip_prone(n, L, M, rng):
    """Positions (Float32) whose Float32 anchor differs from the Float64 one
    on some axis, found by rejection."""
    h32 = np.float32(np.float32(L) / np.float32(M))
    inv_h32 = np.float32(np.float32(1) / h32)
    inv_h64 = 1.0 / (L / M)
    out = []
    while len(out) < n:
        j = rng.integers(M // 2, M, size=4096)
        y = ((j + 0.5) * (L / M) * (1 + rng.normal(0, 2e-7, 4096))).astype(np.float32)
        a32 = np.rint(np.float32(y * inv_h32))
        a64 = np.rint(y.astype(np.float64) * inv_h64)
        out.extend(y[a32 != a64][: n - len(out)])
    return np.array(out, np.float32)


def test_float64_geometry_removes_anchor_flips():
    rng = np.random.default_rng(5)
    L, M, N = 68.9, 128, 400
    Y = (rng.random((N, 3)) * L).astype(np.float32)
    Y[:60, 0] = _flip_prone(60, L, M, rng)
    F = rng.standard_normal((N, 3)).astype(np.float32)
    kw = dict(L=(L,) * 3, R_c=3.0, N=N, kernel_widths_ratio=2.0, viscosity=1.0, num_grid_points=(M,) * 3, M_G=8)
    V64 = O.apply(O.OracleConfig(np.float64, **kw), Y.astype(np.float64), F.astype(np.float64))
    V32 = O.apply(O.OracleConfig(np.float32, **kw), Y, F)
    Vg = O.apply(O.OracleConfig(np.float32, stencil="float64", **kw), Y, F)
    err = lambda a: float(np.linalg.norm(a - V64) / np.linalg.norm(V64))  # noqa: E731
    assert err(V32) > 1e-4           # the reference's Float32 anchors flip
    assert err(Vg) < 2e-6            # Float64 geometry follows Float64
    # in Float64 the option changes nothing but the offset's rounding
    Vg64 = O.apply(O.OracleConfig(np.float64, stencil="float64", **kw), Y.astype(np.float64), F.astype(np.float64))
    assert float(np.linalg.norm(Vg64 - V64) / np.linalg.norm(V64)) < 1e-12
