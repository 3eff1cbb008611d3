"""Host-side checks of the C ABI (no device work, runs without a GPU):

* libffcm_b200.so loads and exports every function include/ffcm_b200.h declares;
* ffcm_validate_config raises exactly where the reference's constructor does
  (src/config.jl:267-312, 341-348), compared with the oracle's restatement;
* ffcm_derive_scalars returns the oracle's derived scalars bit for bit, in
  Float32 and Float64 (src/config.jl:326-359).
"""
import itertools

import numpy as np
import pytest

import ffcm_oracle as O


def test_library_exports_every_declared_symbol(ffcm):
    from ffcm_b200 import _lib
    lib = _lib.load()
    declared = _lib.declared_symbols()
    assert len(declared) >= 20
    missing = [s for s in declared if not hasattr(lib, s)]
    assert missing == []
    assert set(_lib.SIGNATURES) == set(declared)
    assert lib.ffcm_version() >= 100


BASE = dict(L=(8.0, 8.0, 8.0), R_c=1.0, N=4, a=1.0, kernel_widths_ratio=2.0,
            num_grid_points=(16, 16, 16), M_G=8, viscosity=1.0, fft_planning="estimate",
            fft_threads=1)

BAD = [
    dict(R_c=0.0), dict(R_c=-1.0), dict(R_c=float("nan")), dict(L=(0.0, 8.0, 8.0)),
    dict(L=(8.0, -1.0, 8.0)), dict(R_c=4.5), dict(N=0), dict(N=-3), dict(a=2.0),
    dict(kernel_widths_ratio=0.99), dict(M_G=1), dict(M_G=17),
    dict(num_grid_points=(0, 16, 16)), dict(viscosity=0.0), dict(viscosity=-2.0),
    dict(fft_threads=0), dict(num_grid_points=(16, 16, 15)),
    dict(L=(8.0, 8.0, 4.0), R_c=2.5),
]
GOOD = [
    dict(), dict(R_c=4.0), dict(L=(4.0, 6.0, 8.0), num_grid_points=(8, 12, 16)),
    dict(kernel_widths_ratio=1.0), dict(M_G=2), dict(M_G=16), dict(fft_planning="patient"),
    dict(L=(2.0, 2.0, 2.0), num_grid_points=(8, 8, 8)),
]


def _oracle_accepts(T, kw):
    try:
        O.OracleConfig(T, **kw)
        return True
    except O.ArgumentError:
        return False


@pytest.mark.parametrize("T", [np.float32, np.float64])
@pytest.mark.parametrize("over", BAD + GOOD)
def test_validation_matches_reference_rules(ffcm, T, over):
    kw = {**BASE, **over}
    expected_ok = _oracle_accepts(T, kw)
    if expected_ok:
        ffcm.validate_config(T, **kw)
    else:
        with pytest.raises(ffcm.ArgumentError):
            ffcm.validate_config(T, **kw)


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_invalid_planning_and_gpu_only(ffcm, T):
    with pytest.raises(ffcm.ArgumentError):
        ffcm.validate_config(T, **{**BASE, "fft_planning": "fastest"})


CASES = [
    dict(L=(40.0, 40.0, 40.0), R_c=3.0, num_grid_points=(64, 64, 64)),
    dict(L=(275.6, 275.6, 275.6), R_c=3.0, num_grid_points=(512, 512, 512)),
    dict(L=(161.0, 161.0, 161.0), R_c=3.0, num_grid_points=(256, 256, 256)),
    dict(L=(300.0, 300.0, 300.0), R_c=3.0, num_grid_points=(1024, 1024, 1024)),
    dict(L=(4.0, 6.0, 8.0), R_c=1.0, num_grid_points=(8, 12, 16)),
    dict(L=(8.0, 8.0, 8.0), R_c=1.0, num_grid_points=(32, 32, 32)),
    dict(L=(7.0, 5.0, 6.0), R_c=0.7, num_grid_points=(14, 10, 12)),
]


@pytest.mark.parametrize("T", [np.float32, np.float64])
@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("ratio", [1.0, 1.25, 2.0])
def test_derived_scalars_bit_identical(ffcm, T, case, ratio):
    got = ffcm.derive_scalars(T, L=case["L"], R_c=case["R_c"], kernel_widths_ratio=ratio,
                              num_grid_points=case["num_grid_points"])
    Tt = np.dtype(T).type
    ref = O.derive_scalars(Tt, L=tuple(Tt(x) for x in case["L"]), R_c=Tt(case["R_c"]), a=Tt(1),
                           kernel_widths_ratio=Tt(ratio),
                           num_grid_points=case["num_grid_points"])
    assert got["num_cells"] == ref["num_cells"]
    for k in ("cell_size", "inv_cell_size"):
        assert all(Tt(a) == Tt(b) for a, b in zip(got[k], ref[k])), k
    for k in ("sigma", "Sigma", "h", "inv_h"):
        assert Tt(got[k]) == Tt(ref[k]), k


def test_create_requires_gpu_acceleration(ffcm):
    with pytest.raises(ffcm.ArgumentError):
        ffcm.FFCMConfig(np.float32, gpu_acceleration=False, **{k: v for k, v in BASE.items()})
