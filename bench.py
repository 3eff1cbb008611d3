"""Benchmark of the FFCM mobility solve on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: N = 500,000 non-overlapping unit spheres, cubic box L = 275.6
(volume fraction 10%), 512^3 grid, M_G = 8, R_c = 3, Sigma/sigma = 2, mu = 1,
Float32; forces i.i.d. N(0, 1). Synthetic seeded inputs (no dataset).

A step is one mobility solve V = M(Y) F. `value` is particles/s with Y and F
already resident in HBM; `e2e` is the same metric through the public API with
pinned host buffers (H2D of Y and F, D2H of V inside every timed step). The
working set (three 512^3 grids, ~5 GB) is far larger than the 126 MB L2, so
every step streams from HBM. With --gpus N > 1 (torchrun) each rank solves
its own replica of the system ("replicas only": the single-system path has no
data exchange); the time is the max over ranks.

--impl reference times the reference's CPU algorithm (the oracle restatement;
the Julia reference cannot run on this machine) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT / "oracle"))

METRIC = "particles/s per mobility solve (N=500k, 512^3, Float32)"
UNIT = "particles/s"
WORK = dict(L=275.6, N=500_000, M=512, M_G=8, R_c=3.0, ratio=2.0, mu=1.0, seed=2024 + 1)


def config_kwargs():
    w = WORK
    return dict(L=(w["L"],) * 3, R_c=w["R_c"], N=w["N"], kernel_widths_ratio=w["ratio"],
                viscosity=w["mu"], num_grid_points=(w["M"],) * 3, M_G=w["M_G"])


def workload_config():
    w = WORK
    return {"workload": f"plain FFCM mobility, N={w['N']}, L={w['L']}, grid {w['M']}^3, "
                        f"M_G={w['M_G']}, R_c={w['R_c']}, Sigma/sigma={w['ratio']}, Float32",
            "N": w["N"], "grid": [w["M"]] * 3, "M_G": w["M_G"],
            "l2": "working set ~5 GB >> 126 MB L2 (grids rewritten every step); no flush needed"}


def make_inputs():
    from fixtures import nonoverlapping_uniform
    w = WORK
    Y = nonoverlapping_uniform(w["N"], w["L"], w["seed"]).astype(np.float32)
    F = np.random.default_rng(w["seed"]).standard_normal((w["N"], 3)).astype(np.float32)
    return Y, F


def algorithmic_bytes(T_bytes=4):
    """Compulsory HBM traffic per solve and per stage (each input read once,
    each output written once)."""
    w = WORK
    N, M = w["N"], w["M"]
    grid = 3 * M ** 3 * T_bytes
    spec = 3 * (M // 2 + 1) * M * M * 2 * T_bytes
    ncell = int(np.floor(np.float32(w["L"]) / np.float32(w["R_c"]))) ** 3
    per = {
        "cell_list": N * (12 + 12 + 4 + 4 + 24) + 8 * ncell,
        "spread": grid + 24 * N,
        "fft_x_fwd": grid + spec,
        "fft_y_fwd": 2 * spec,
        "fft_z_stokes": 2 * spec,
        "fft_y_inv": 2 * spec,
        "fft_x_inv": spec + grid,
        "interpolate": grid + 28 * N,
        "correct": 36 * N,
    }
    solve = per["cell_list"] + per["spread"] + 2 * grid + per["interpolate"] + per["correct"]
    return per, solve


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "").strip()
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        self.dev = ids[device_index] if device_index < len(ids) else str(device_index)
        self.proc = None
        self.path = Path(f"/tmp/ffcm_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(stage):
    """Per-launch DRAM bytes of a stage's kernel from the committed ncu summary."""
    p = ROOT / "profiles" / "ncu_traffic_c2.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 2 and parts[0] == stage:
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


def cpu_baseline_run(Y, F, threads):
    """One full solve of the workload by the CPU oracle (particle loops serial as
    in the reference, FFT with `threads` workers as fft_threads)."""
    import ffcm_oracle as O
    cfg = O.OracleConfig(np.float32, **config_kwargs(), fft_threads=threads)
    V = np.zeros_like(Y)
    t0 = time.perf_counter()
    O.mobility(V, cfg, Y, F)
    return time.perf_counter() - t0


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    import ffcm_oracle as O  # noqa: F401
    Y, F = make_inputs()
    threads = os.cpu_count() or 1
    # each step is one full solve (~tens of seconds); bound the run to a few minutes
    warm = min(args.warmup, 1)
    steps = min(args.steps, 3)
    for _ in range(warm):
        cpu_baseline_run(Y, F, threads)
    ts = [cpu_baseline_run(Y, F, threads) for _ in range(steps)]
    sec = float(np.mean(ts))
    value = WORK["N"] / sec
    sample = (f"{warm} warm-up + {steps} timed full solves of the workload by the C/pocketfft "
              f"restatement of the reference CPU path (Julia is not installed)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, world, local_rank):
    import torch
    import importlib.util

    pkg = ROOT / "ffcm.jl_b200"
    spec = importlib.util.spec_from_file_location("ffcm_b200", pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    ffcm = importlib.util.module_from_spec(spec)
    sys.modules["ffcm_b200"] = ffcm
    spec.loader.exec_module(ffcm)

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)

    Y, F = make_inputs()
    N = WORK["N"]
    cfg = ffcm.FFCMConfig(np.float32, device=local_rank, **config_kwargs())
    Yd = torch.from_numpy(Y).to(dev)
    Fd = torch.from_numpy(F).to(dev)
    Vd = torch.empty_like(Yd)
    stream = torch.cuda.current_stream(dev)

    def barrier():
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
            torch.cuda.synchronize(dev)

    def step():
        ffcm.mobility(Vd, cfg, Yd, Fd)

    for _ in range(args.warmup):
        step()
    barrier()

    # ---- main timed region: device-resident inputs --------------------------
    launches0 = cfg.launch_count()
    with ClockSampler(local_rank) as clk:
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        barrier()
    launches = cfg.launch_count() - launches0
    ms = e0.elapsed_time(e1) / args.steps

    # ---- per-stage CUDA events over a second timed pass ----------------------
    cfg.profile_begin()
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize(dev)
    stages = cfg.profile_end()

    # ---- end to end through the public API with pinned host buffers ---------
    Yh = torch.from_numpy(Y).pin_memory()
    Fh = torch.from_numpy(F).pin_memory()
    Vh = torch.empty_like(Yh).pin_memory()
    for _ in range(max(1, args.warmup)):
        ffcm.mobility(Vh, cfg, Yh, Fh, stream=stream)
    barrier()
    h0 = torch.cuda.Event(enable_timing=True)
    h1 = torch.cuda.Event(enable_timing=True)
    h0.record(stream)
    for _ in range(args.steps):
        ffcm.mobility(Vh, cfg, Yh, Fh, stream=stream)
    h1.record(stream)
    barrier()
    ms_e2e = h0.elapsed_time(h1) / args.steps

    # max over ranks
    if dist is not None:
        t = torch.tensor([ms, ms_e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_e2e = float(t[0]), float(t[1])

    if rank == 0:
        value = world * N / (ms / 1e3)
        e2e_value = world * N / (ms_e2e / 1e3)
        per, solve_bytes = algorithmic_bytes()
        peak, peak_kind = measured_peak_hbm()
        stage_ms = {k: v[0] / max(v[1], 1) for k, v in stages.items() if v[1] > 0}
        kernel_stages = [k for k in per if k in stage_ms]
        dom = max(kernel_stages, key=lambda k: stage_ms[k])
        achieved = per[dom] / (stage_ms[dom] / 1e3) / 1e9
        traffic = ncu_traffic(dom)
        # CPU baseline: one full solve of the workload by the oracle on the host
        cpu_threads = os.cpu_count() or 1
        if args.skip_cpu_baseline:
            cpu = None
        else:
            sec = cpu_baseline_run(Y, F, cpu_threads)
            cpu = {"value": N / sec, "unit": UNIT, "cores": cpu_threads, "kind": "port",
                   "sample": "one full solve of the workload by the C/pocketfft restatement of "
                             "the reference CPU path; particle loops serial as in the reference, "
                             f"FFT on {cpu_threads} threads (fft_threads)"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {**workload_config(),
                                            "parallelism": "replicas" if world > 1 else "single"},
            "e2e": {"value": e2e_value, "unit": UNIT, "ms_per_step": ms_e2e,
                    "h2d_bytes_per_step": int(Yh.numel() * 4 + Fh.numel() * 4),
                    "d2h_bytes_per_step": int(Vh.numel() * 4)},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": traffic,
                         "algorithmic_bytes_per_launch": per[dom]},
            "solve_roofline": {"algorithmic_bytes": solve_bytes,
                               "achieved_GBs": solve_bytes / (ms / 1e3) / 1e9,
                               "frac": solve_bytes / (ms / 1e3) / 1e9 / peak},
            "stage_ms": {k: round(v, 4) for k, v in stage_ms.items()},
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
        }
        print(json.dumps(line), flush=True)
    cfg.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--skip-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", args.gpus if args.gpus == 1 else 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
