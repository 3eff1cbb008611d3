"""Every launch variant the autotuner can choose computes the same solve.

The autotuner keeps whichever y-pass, z-pass and kx-chunk variant is fastest
on the machine at hand, so a parity test only ever sees the winner. Here
each variant is pinned in turn (FFCM_FORCE_Y / FFCM_FORCE_Z = "kind,B",
FFCM_FORCE_CHUNK = columns) and the solve compared with the oracle."""
import os

import numpy as np
import pytest

import ffcm_oracle as O
from fixtures import nonoverlapping_uniform
from gpu_helpers import rel_l2

pytestmark = pytest.mark.gpu

CASES = {"64^3": dict(L=(40.0,) * 3, N=2000, M=(64, 64, 64)),
         "128^3": dict(L=(60.0,) * 3, N=5000, M=(128, 128, 128)),
         "64x32x32": dict(L=(32.0, 16.0, 16.0), N=300, M=(64, 32, 32)),
         # lines of 1024 along z, y and x (the last through the slab kernels at
         # x length 1024), spacing and density of the 64^3 case
         "64x64x1024": dict(L=(40.0, 40.0, 640.0), N=32000, M=(64, 64, 1024)),
         "64x1024x64": dict(L=(40.0, 640.0, 40.0), N=32000, M=(64, 1024, 64)),
         "1024x64x64": dict(L=(640.0, 40.0, 40.0), N=32000, M=(1024, 64, 64)),
         # lines of 512 and 256 along y (also the three-plane y pass)
         "64x512x64": dict(L=(40.0, 320.0, 40.0), N=16000, M=(64, 512, 64)),
         "64x256x64": dict(L=(40.0, 160.0, 40.0), N=8000, M=(64, 256, 64)),
         # lines of 256 and 512 along z (the in-place wide-tile z pass)
         "64x64x256": dict(L=(40.0, 40.0, 160.0), N=8000, M=(64, 64, 256)),
         "64x64x512": dict(L=(40.0, 40.0, 320.0), N=16000, M=(64, 64, 512))}
Y_VARIANTS = [(k, B) for k in (0, 1, 2, 3) for B in (2, 4, 8, 16)]
Z_VARIANTS = [(k, B) for k in (0, 1, 2, 3, 4) for B in (2, 4, 8, 16)]


def _solve(ffcm, T, case, env):
    c = CASES[case]
    kw = dict(L=c["L"], R_c=3.0 if case != "64x32x32" else 2.0, N=c["N"], kernel_widths_ratio=2.0,
              viscosity=1.0, num_grid_points=c["M"], M_G=8)
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        cfg = ffcm.FFCMConfig(T, **kw)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    rng = np.random.default_rng(c["N"])
    Y = nonoverlapping_uniform(c["N"], c["L"], 3).astype(T)
    F = rng.standard_normal((c["N"], 3)).astype(T)
    V = np.empty_like(Y)
    ffcm.mobility(V, cfg, Y, F)
    ora = O.OracleConfig(T, **kw)
    return rel_l2(V, O.apply(ora, Y, F))


def _check(ffcm, T, case, env):
    try:
        err = _solve(ffcm, T, case, env)
    except ffcm.ArgumentError:
        pytest.skip("variant not available for this configuration")
    assert err < (1e-5 if T == np.float32 else 1e-10), (env, err)


@pytest.mark.parametrize("T", [np.float32, np.float64])
@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("kind,B", Y_VARIANTS)
def test_y_variant(ffcm, T, case, kind, B):
    _check(ffcm, T, case, {"FFCM_FORCE_Y": f"{kind},{B}", "FFCM_FORCE_CHUNK": "0"})


@pytest.mark.parametrize("T", [np.float32, np.float64])
@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("kind,B", Z_VARIANTS)
def test_z_variant(ffcm, T, case, kind, B):
    _check(ffcm, T, case, {"FFCM_FORCE_Z": f"{kind},{B}", "FFCM_FORCE_CHUNK": "0"})


# (y, z) variants pinned with chunking, so that which chunk widths apply does
# not depend on what the autotuner happens to pick
CHUNK_PINS = {"register": ("0,8", "0,8"), "pipelined": ("1,8", "1,4"), "tma": ("2,8", "3,8"),
              "tma3": ("3,4", "3,8")}


@pytest.mark.parametrize("T", [np.float32, np.float64])
@pytest.mark.parametrize("case", ["64^3", "128^3", "64x256x64"])
@pytest.mark.parametrize("chunk", [8, 16, 32])
@pytest.mark.parametrize("pin", list(CHUNK_PINS))
def test_chunked_yz(ffcm, T, case, chunk, pin):
    y, z = CHUNK_PINS[pin]
    _check(ffcm, T, case, {"FFCM_FORCE_CHUNK": str(chunk), "FFCM_FORCE_Y": y, "FFCM_FORCE_Z": z})
