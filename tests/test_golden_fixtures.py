"""The committed golden fixtures are reproduced by the oracle (guards both the
fixtures and the oracle against drift). CPU only."""
from pathlib import Path

import numpy as np
import pytest

import ffcm_oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("name", ["standard_random256", "uniform_N2000_64"])
@pytest.mark.parametrize("tag,T", [("f32", np.float32), ("f64", np.float64)])
def test_oracle_reproduces_fixture(name, tag, T):
    z = np.load(GOLDEN / f"{name}.npz")
    L, N, M, MG, Rc, ratio = z["meta"]
    cfg = O.OracleConfig(T, L=(L, L, L), R_c=Rc, N=int(N), kernel_widths_ratio=ratio,
                         viscosity=1.0, num_grid_points=(int(M),) * 3, M_G=int(MG))
    V = O.apply(cfg, z[f"{tag}_Y"], z[f"{tag}_F"])
    assert (cfg.original_index == z[f"{tag}_original_index"]).all()
    assert (cfg.cell_start == z[f"{tag}_cell_start"]).all()
    assert (cfg.cell_end == z[f"{tag}_cell_end"]).all()
    # pocketfft's threaded and serial paths agree to round-off, not bitwise
    np.testing.assert_allclose(V, z[f"{tag}_V"], rtol=1e-5 if T == np.float32 else 1e-12,
                               atol=1e-7 if T == np.float32 else 1e-15)


def test_fixture_f32_close_to_f64():
    z = np.load(GOLDEN / "uniform_N2000_64.npz")
    v32, v64 = z["f32_V"].astype(np.float64), z["f64_V"]
    assert np.linalg.norm(v32 - v64) / np.linalg.norm(v64) < 1e-5
