"""Launch-shape wisdom on the GPU: a configuration reports the variant it
uses, the autotuner's choices show up in the exported wisdom, an imported
choice is taken by the next configuration of that shape (and the solve still
matches the oracle), and an imported choice naming a variant the shape cannot
run is ignored in favour of the autotuner."""
import numpy as np
import pytest

import ffcm_oracle as O
from fixtures import nonoverlapping_uniform
from gpu_helpers import both, kw_of, rel_l2

pytestmark = pytest.mark.gpu

# an unusual shape so no other test shares its wisdom entry: x 64, y 32, z 128
L3, M3, N = (40.0, 20.0, 80.0), (64, 32, 128), 1500


def _sms():
    import torch
    return torch.cuda.get_device_properties(0).multi_processor_count


def _solve(ffcm, cfg, ora, seed):
    Y = nonoverlapping_uniform(N, L3, seed=seed).astype(np.float32)
    F = np.random.default_rng(seed).standard_normal((N, 3)).astype(np.float32)
    V = np.empty_like(Y)
    ffcm.mobility(V, cfg, Y, F)
    return rel_l2(V, O.apply(ora, Y, F))


def test_autotuned_choice_is_exported(ffcm):
    cfg, _ = both(ffcm, np.float32, **kw_of(40.0, 2000, 64, R_c=3.0))
    t = cfg.tuning()
    line = (f"ffcm-wisdom-2 0 4 64 64 64 {_sms()} {t['y_kind']} {t['y_columns']} {t['y_grid']} "
            f"{t['z_kind']} {t['z_columns']} {t['z_grid']} {t['kx_chunk']}")
    assert line in ffcm.wisdom_export().splitlines()


def test_imported_choice_is_used_and_correct(ffcm):
    # TMA y and z passes with 8 columns per tile and grids the autotuner would
    # never pick (it sizes persistent grids by occupancy x SM count)
    ffcm.wisdom_import(f"ffcm-wisdom-2 0 4 64 32 128 {_sms()} 2 8 37 3 8 41 0")
    cfg, ora = both(ffcm, np.float32, **kw_of(L3, N, M3, R_c=3.0))
    assert cfg.tuning() == dict(y_kind=2, y_columns=8, y_grid=37, z_kind=3, z_columns=8, z_grid=41,
                                kx_chunk=0)
    assert _solve(ffcm, cfg, ora, 5) < 1e-5


def test_import_for_another_gpu_model_is_not_used(ffcm):
    # the same ordinal and shape (a shape of its own: x 64, y 64, z 32), but a
    # GPU with one SM more: the key differs, so the configuration times its
    # own variants instead of taking grids sized for that other GPU
    L4, M4 = (40.0, 40.0, 20.0), (64, 64, 32)
    ffcm.wisdom_import(f"ffcm-wisdom-2 0 4 64 64 32 {_sms() + 1} 2 8 37 3 8 41 0")
    cfg, ora = both(ffcm, np.float32, **kw_of(L4, N, M4, R_c=3.0))
    t = cfg.tuning()
    assert (t["y_grid"], t["z_grid"]) != (37, 41)
    Y = nonoverlapping_uniform(N, L4, seed=7).astype(np.float32)
    F = np.random.default_rng(7).standard_normal((N, 3)).astype(np.float32)
    V = np.empty_like(Y)
    ffcm.mobility(V, cfg, Y, F)
    assert rel_l2(V, O.apply(ora, Y, F)) < 1e-5


def test_unrunnable_import_is_ignored(ffcm):
    # 3 columns per tile exists for no pass: the configuration times its own
    ffcm.wisdom_import(f"ffcm-wisdom-2 0 4 64 32 128 {_sms()} 2 3 37 3 3 41 0")
    cfg, ora = both(ffcm, np.float32, **kw_of(L3, N, M3, R_c=3.0))
    t = cfg.tuning()
    assert t["y_columns"] != 3 and t["z_columns"] != 3
    assert _solve(ffcm, cfg, ora, 6) < 1e-5
    # and its own choice replaced the unrunnable one
    assert any(l.startswith(f"ffcm-wisdom-2 0 4 64 32 128 {_sms()} ") and " 3 37 " not in l
               for l in ffcm.wisdom_export().splitlines())
