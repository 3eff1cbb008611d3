"""Generate the golden fixtures under tests/golden/ from the CPU oracle.

    python tests/golden/make_golden.py

Each fixture holds seeded inputs and the oracle's outputs (cell list and
velocities) for one configuration, in the reference layouts (1-based index
buffers, (N, 3) = Julia 3xN). The reference itself (Julia) cannot run in this
environment; the oracle that produced these files is pinned by the
reference's own known-answer tests (tests/test_oracle_*.py).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent / "oracle"))
sys.path.insert(0, str(HERE.parent))

import ffcm_oracle as O  # noqa: E402
from fixtures import nonoverlapping_uniform, random_cloud  # noqa: E402

CASES = {
    # test/cuda/test_gpu_mobility.jl random cloud: L=8, 16^3, M_G=8, R_c=1, ratio 2
    "standard_random256": dict(L=8.0, N=256, M=16, M_G=8, R_c=1.0, ratio=2.0, seed=0xC7A0,
                               kind="random"),
    # the 64^3 workload: L=40, N=2000 non-overlapping, M_G=8, R_c=3, ratio 2, N(0,1) forces
    "uniform_N2000_64": dict(L=40.0, N=2000, M=64, M_G=8, R_c=3.0, ratio=2.0, seed=2024 + 0,
                        kind="nonoverlap"),
}


def inputs(case):
    if case["kind"] == "random":
        Y, F = random_cloud(np.float64, case["N"], (case["L"],) * 3, case["seed"])
        return Y.astype(np.float64), F.astype(np.float64)
    rng = np.random.default_rng(case["seed"])
    Y = nonoverlapping_uniform(case["N"], case["L"], case["seed"])
    F = rng.standard_normal((case["N"], 3))
    return Y, F


def run(case, T):
    Y, F = inputs(case)
    Y, F = Y.astype(T), F.astype(T)
    cfg = O.OracleConfig(T, L=(case["L"],) * 3, R_c=case["R_c"], N=case["N"],
                         kernel_widths_ratio=case["ratio"], viscosity=1.0,
                         num_grid_points=(case["M"],) * 3, M_G=case["M_G"])
    V = O.apply(cfg, Y, F)
    return dict(Y=Y, F=F, V=V, original_index=cfg.original_index.copy(),
                cell_start=cfg.cell_start.copy(), cell_end=cfg.cell_end.copy(),
                cell_hash=cfg.cell_hash.copy())


def main():
    for name, case in CASES.items():
        out = {}
        for T, tag in ((np.float32, "f32"), (np.float64, "f64")):
            r = run(case, T)
            for k, v in r.items():
                out[f"{tag}_{k}"] = v
        meta = np.array([case["L"], case["N"], case["M"], case["M_G"], case["R_c"], case["ratio"]])
        np.savez_compressed(HERE / f"{name}.npz", meta=meta, **out)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
