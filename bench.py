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

--workload selects the other measured configurations: `batched` (64
suspensions x 16 right-hand sides in one graph launch), `adjoint` (objective
gradient at N=100k, 256^3), `resistance` (conjugate-gradient resistance solve
on the 512^3 system), `clustered` (N=2M in 2,000 Gaussian clusters, 1024^3),
`split` (the 512^3 system as one system over all --gpus, by z slabs:
strong scaling, two spectrum transposes over NCCL per solve).
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


GRID = None   # optional (Mx, My, Mz) override for small profiling cases


def work_geometry():
    """(L, N, M) of the workload; a --grid override keeps the spacing
    h = 275.6/512 and the particle density, scaling the box and N."""
    w = WORK
    if GRID is None:
        return (w["L"],) * 3, w["N"], (w["M"],) * 3
    h = w["L"] / w["M"]
    L = tuple(h * m for m in GRID)
    N = int(round(w["N"] * np.prod(GRID) / w["M"] ** 3))
    return L, N, tuple(GRID)


def config_kwargs():
    w = WORK
    L, N, M = work_geometry()
    return dict(L=L, R_c=w["R_c"], N=N, kernel_widths_ratio=w["ratio"],
                viscosity=w["mu"], num_grid_points=M, M_G=w["M_G"])


def workload_config():
    w = WORK
    L, N, M = work_geometry()
    return {"workload": f"plain FFCM mobility, N={N}, L={L[0] if len(set(L)) == 1 else L}, grid "
                        f"{M[0] if len(set(M)) == 1 else M}^3, M_G={w['M_G']}, R_c={w['R_c']}, "
                        f"Sigma/sigma={w['ratio']}, Float32",
            "N": N, "grid": list(M), "M_G": w["M_G"],
            "l2": "working set ~5 GB >> 126 MB L2 (grids rewritten every step); no flush needed"}


def make_inputs():
    from fixtures import nonoverlapping_uniform
    w = WORK
    L, N, _ = work_geometry()
    Y = nonoverlapping_uniform(N, L, w["seed"]).astype(np.float32)
    F = np.random.default_rng(w["seed"]).standard_normal((N, 3)).astype(np.float32)
    return Y, F


def algorithmic_bytes(T_bytes=4, geometry=None):
    """Compulsory HBM traffic per solve and per stage (each input read once,
    each output written once). geometry = (L, N, M) of another workload (the
    plain 512^3 one by default)."""
    w = WORK
    L, N, M3 = work_geometry() if geometry is None else geometry
    grid = 3 * int(np.prod(M3)) * T_bytes
    spec = 3 * (M3[0] // 2 + 1) * M3[1] * M3[2] * 2 * T_bytes
    ncell = int(np.prod([max(int(np.floor(np.float32(x) / np.float32(w["R_c"]))), 3) for x in L]))
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
                 "-lms", "50"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
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
    p = ROOT / "profiles" / "ncu_traffic_plain_N500k_512cubed.txt"
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


def cpu_baseline_run(Y, F, threads, keep=None):
    """One full solve of the workload by the CPU oracle (particle loops serial as
    in the reference, FFT with `threads` workers as fft_threads). With `keep`
    (a list), the oracle's velocities are appended to it."""
    import ffcm_oracle as O
    cfg = O.OracleConfig(np.float32, **config_kwargs(), fft_threads=threads)
    V = np.zeros_like(Y)
    t0 = time.perf_counter()
    O.mobility(V, cfg, Y, F)
    sec = time.perf_counter() - t0
    if keep is not None:
        keep.append(V)
    return sec


def accuracy_report(V, Y, F, V32, threads, V_comp=None):
    """Errors of the GPU velocities against the oracle: rel-L2 and max-abs
    against the Float64 restatement, rel-L2 against the Float32 one; with
    V_comp, the same for the solve with Float64 stencil geometry."""
    import ffcm_oracle as O
    cfg = O.OracleConfig(np.float64, **config_kwargs(), fft_threads=threads)
    V64 = O.apply(cfg, Y.astype(np.float64), F.astype(np.float64))
    V = np.asarray(V, np.float64)
    d64 = V - V64
    comp = None
    if V_comp is not None:
        dc = np.asarray(V_comp, np.float64) - V64
        comp = {"rel_l2_vs_oracle_f64": float(np.linalg.norm(dc) / np.linalg.norm(V64)),
                "max_abs_vs_oracle_f64": float(np.abs(dc).max()),
                "rel_l2_vs_oracle_f32": float(np.linalg.norm(np.asarray(V_comp, np.float64) - V32)
                                              / np.linalg.norm(V32)),
                "how": "ffcm_set_stencil(FFCM_STENCIL_FLOAT64): stencil anchors and offsets from the "
                       "double box spacing, weights in Float32; same cell list, not the reference's "
                       "Float32 arithmetic"}
    return {"stencil_float64": comp,
            "rel_l2_vs_oracle_f64": float(np.linalg.norm(d64) / np.linalg.norm(V64)),
            "max_abs_vs_oracle_f64": float(np.abs(d64).max()),
            "max_abs_oracle_f64": float(np.abs(V64).max()),
            "rel_l2_vs_oracle_f32": float(np.linalg.norm(V - V32) / np.linalg.norm(V32)),
            # the Float32 restatement's own distance from Float64: the floor any
            # Float32 implementation of the reference sits at on this workload
            "oracle_f32_rel_l2_vs_oracle_f64": float(np.linalg.norm(np.asarray(V32, np.float64) - V64)
                                                     / np.linalg.norm(V64)),
            "targets": "rel-L2 <= 1e-4 vs Float64, <= 1e-5 vs the Float32 restatement"}


def run_reference(args, rank, world):
    """The reference's CPU algorithm (the oracle restatement; Julia is not
    installed here) on the host cores, on the same workload as --workload."""
    if rank != 0:
        return 0
    import ffcm_oracle as O
    threads = os.cpu_count() or 1
    # each step is one full evaluation (seconds to tens of seconds): bound the run
    warm = min(args.warmup, 1)
    steps = min(args.steps, 3)
    if args.workload == "clustered":
        print(json.dumps({"impl": "reference", "unavailable":
                          "clustered 1024^3 workload: the CPU restatement's serial pair correction over "
                          "the dense clusters does not fit a bounded sample; see the plain workload"}), flush=True)
        return 0
    if args.workload == "adjoint":
        Y, F, Yp = adjoint_inputs()
        cfg = O.OracleConfig(np.float32, **adjoint_kwargs(), fft_threads=threads)
        Vt = O.apply(cfg, Yp, F)
        fn = lambda: cpu_adjoint_run(Y, F, Vt, threads)  # noqa: E731
        units, unit = Y.shape[0], "particles/s"
        metric = "particles/s per gradient evaluation (J, dJ/dY, dJ/dF; N=100k, 256^3, Float32)"
        config = adjoint_config()
        sample = (f"{warm} warm-up + {steps} timed objective-gradient evaluations of the workload by "
                  "the C/pocketfft restatement (forward, residual, pullback)")
    elif args.workload == "resistance":
        Y, V = resistance_inputs()
        cfg = O.OracleConfig(np.float32, **config_kwargs(), fft_threads=threads)

        def fn():
            t0 = time.perf_counter()
            O.cg(cfg, Y, V, maxiter=1)
            return time.perf_counter() - t0

        units, unit, metric, config = Y.shape[0], "particles/s", RES_METRIC, resistance_config()
        sample = (f"{warm} warm-up + {steps} timed CG iterations (maxiter = 1: one operator application "
                  "and the vector updates) of the workload by the C/pocketfft restatement; "
                  "particles/s per CG iteration of that sample")
    elif args.workload == "batched":
        from fixtures import nonoverlapping_uniform
        b = BATCH
        systems = batched_systems()
        order = np.argsort([s_["N"] for s_ in systems])
        pick = [int(order[k]) for k in range(3, len(systems), 8)]  # 8 systems, stratified by N
        rng = np.random.default_rng(b["seed"] + 1)
        cases = []
        for i in pick:
            s_ = systems[i]
            cfg = O.OracleConfig(np.float32, L=s_["L"], R_c=s_["R_c"], N=s_["N"],
                                 num_grid_points=s_["num_grid_points"], kernel_widths_ratio=b["ratio"],
                                 M_G=b["M_G"], viscosity=b["mu"], fft_threads=threads)
            y = nonoverlapping_uniform(s_["N"], s_["L"][0], b["seed"] + 10 + i).astype(np.float32)
            cases.append((cfg, y, rng.standard_normal((s_["N"], 3)).astype(np.float32)))

        def fn():
            t0 = time.perf_counter()
            for cfg, y, f in cases:
                O.apply(cfg, y, f)
            return time.perf_counter() - t0

        units, unit = len(cases), "solves/s"
        metric = f"solves/s, batched form ({b['nsys']} systems x {b['nrhs']} right-hand sides)"
        config = {"workload": "batched FFCM mobility (see the ours line); reference solves systems "
                              "one at a time", "total_particles": int(sum(s_["N"] for s_ in systems))}
        sample = (f"{warm} warm-up + {steps} timed passes over 8 of the 64 systems (stratified by N), "
                  "one right-hand side each, by the C/pocketfft restatement; solves/s of that sample")
    else:
        Y, F = make_inputs()
        fn = lambda: cpu_baseline_run(Y, F, threads)  # noqa: E731
        units, unit, metric, config = Y.shape[0], UNIT, METRIC, workload_config()
        sample = (f"{warm} warm-up + {steps} timed full solves of the workload by the C/pocketfft "
                  f"restatement of the reference CPU path (Julia is not installed)")
    if "parallelism" not in config:
        # the same key as the GPU arm's line for this workload and world size
        par = "replicas" if world > 1 else "single"
        if args.workload == "batched" and world > 1:
            par = "systems sharded across ranks"
        config = {**config, "parallelism": par}
    for _ in range(warm):
        fn()
    ts = [fn() for _ in range(steps)]
    sec = float(np.mean(ts))
    value = units / sec
    line = {"impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config,
            "cpu_baseline": {"value": value, "unit": unit, "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def secondary_workloads(args, local_rank):
    """Batched, adjoint, clustered and resistance measurements for the
    single-GPU line."""
    import copy
    out = {}
    keep = {
        "batched": ("metric", "value", "unit", "ms_per_step", "steps", "warmup", "config", "plain_looped",
                    "speedup_vs_plain_looped", "e2e", "roofline", "clocks", "gpu_launches", "result_checksum"),
        "adjoint": ("metric", "value", "unit", "ms_per_step", "steps", "warmup", "config", "forward_ms",
                    "checkpointed_forward_ms", "pullback_ms", "pullback_cost_vs_forward",
                    "gradient_step_cost_vs_forward", "e2e", "roofline", "pullback_stage_ms", "clocks",
                    "gpu_launches"),
        "clustered": ("metric", "value", "unit", "ms_per_step", "steps", "warmup", "config",
                      "fixed_position_operator_ms_per_rhs", "gradient_ms_per_rhs", "stage_ms", "tuning", "e2e",
                      "roofline", "clocks", "gpu_launches"),
        "resistance": ("metric", "value", "unit", "ms_per_step", "steps", "warmup", "config", "iterations",
                       "solves_per_s", "ms_per_iteration", "apply_ms", "cg_overhead_per_iteration_ms", "e2e",
                       "roofline", "iteration_roofline", "clocks", "gpu_launches"),
    }
    runs = (("batched", measure_batched, 10), ("adjoint", measure_adjoint, 10), ("clustered", measure_clustered, 3),
            ("resistance", lambda *a: measure_resistance(*a)[0], 2))
    for name, fn, steps in runs:
        a = copy.copy(args)
        a.steps, a.warmup, a.skip_cpu_baseline = steps, 3, True
        try:
            line = fn(a, 0, 1, local_rank)
            out[name] = {k: line[k] for k in keep[name] if k in line}
        except Exception as e:   # a failing secondary workload must not hide the headline
            out[name] = {"error": f"{type(e).__name__}: {e}"}
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    ffcm = _load_product()

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)

    Y, F = make_inputs()
    N = Y.shape[0]
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
    tuning = cfg.tuning()

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
        accuracy = None
        if args.skip_cpu_baseline:
            cpu = None
        else:
            kept = []
            sec = cpu_baseline_run(Y, F, cpu_threads, keep=kept)
            # the reference's default, fft_threads = 1: everything on one core
            sec1 = cpu_baseline_run(Y, F, 1)
            cpu = {"value": N / sec, "unit": UNIT, "cores": cpu_threads, "kind": "port",
                   "sample": "one full solve of the workload by the C/pocketfft restatement of "
                             "the reference CPU path; particle loops serial as in the reference, "
                             f"FFT on {cpu_threads} threads (fft_threads)",
                   "single_core": {"value": N / sec1, "unit": UNIT, "cores": 1,
                                   "sample": "the same solve with fft_threads = 1, the reference's default"}}
            # the same solve with Float64 stencil geometry, for the Float64
            # comparison (not timed)
            cfg.stencil = "float64"
            Vc = np.empty_like(Y)
            ffcm.mobility(Vc, cfg, Y, F)
            cfg.stencil = "reference"
            accuracy = accuracy_report(Vh.numpy(), Y, F, kept[0], cpu_threads, V_comp=Vc)
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
            "tuning": tuning,
            "cpu_baseline": cpu,
            "accuracy": accuracy,
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
        }
    cfg.close()
    if rank == 0 and world == 1 and not args.no_extras:
        # the secondary workloads on the same box, each with its own CUDA-event
        # time, clocks and roofline, at reduced step counts
        line.update(secondary_workloads(args, local_rank))
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


BATCH = dict(nsys=64, nrhs=16, Nmin=2000, Nmax=64000, phi=0.1, h0=0.54, Mmin=64, Mmax=256,
             R_c=3.0, M_G=8, ratio=2.0, mu=1.0, seed=2024 + 2)


def batched_systems():
    """64 suspensions: N log-uniform in [2k, 64k], cubic box at 10% volume
    fraction, grid the power of two nearest (in log) to L / 0.54, clamped to
    [64, 256] (tests/fixtures.py: batched_systems, shared with the tests)."""
    from fixtures import batched_systems as make
    b = BATCH
    return make(nsys=b["nsys"], Nmin=b["Nmin"], Nmax=b["Nmax"], phi=b["phi"], h0=b["h0"], Mmin=b["Mmin"],
                Mmax=b["Mmax"], R_c=b["R_c"], seed=b["seed"])


def shard_systems(systems, world):
    """Greedy longest-processing-time assignment of systems to ranks by a cost
    model (particles x stencil + grid x log grid)."""
    cost = [s["N"] * 512 + 3 * np.prod(s["num_grid_points"]) * np.log2(np.prod(s["num_grid_points"]))
            for s in systems]
    order = np.argsort(cost)[::-1]
    load = [0.0] * world
    owner = [0] * len(systems)
    for i in order:
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += cost[i]
    return owner


def stage_roofline(stage_ms, geometry):
    """Roofline of the slowest stage of a solve of the given geometry."""
    per, _ = algorithmic_bytes(geometry=geometry)
    peak, peak_kind = measured_peak_hbm()
    ks = [k for k in per if k in stage_ms]
    if not ks:
        return None
    dom = max(ks, key=lambda k: stage_ms[k])
    ach = per[dom] / (stage_ms[dom] / 1e3) / 1e9
    return {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "peak_source": peak_kind, "traffic": None, "algorithmic_bytes_per_launch": per[dom]}


def batched_roofline(systems, nrhs, ms):
    """Whole-batch algorithmic bytes (every system's solve per right-hand side)
    over the batch time, against the measured HBM peak."""
    peak, peak_kind = measured_peak_hbm()
    total = sum(nrhs * algorithmic_bytes(geometry=(s["L"], s["N"], s["num_grid_points"]))[1] for s in systems)
    ach = total / (ms / 1e3) / 1e9
    return {"bound": "hbm", "kernel": "whole batch", "achieved": ach, "peak": peak, "unit": "GB/s",
            "frac": ach / peak, "peak_source": peak_kind, "traffic": None, "algorithmic_bytes_per_launch": total}


def gather_system_results(mine, parts, nsys, dist, rank):
    """Bring every rank's per-system results to rank 0.

    mine: the global indices of this rank's systems; parts: their results, in
    the same order (any picklable values, e.g. lists of per-right-hand-side
    arrays). Returns the list of all nsys results in global system order on
    rank 0 (None elsewhere). With dist None (one rank) it only reorders."""
    if dist is None:
        out = [None] * nsys
        for i, v in zip(mine, parts):
            out[i] = v
        return out
    world = dist.get_world_size()
    got = [None] * world
    dist.all_gather_object(got, list(zip(mine, parts)))
    if rank != 0:
        return None
    out = [None] * nsys
    for rank_items in got:
        for i, v in rank_items:
            if out[i] is not None:
                raise RuntimeError(f"system {i} was solved by two ranks")
            out[i] = v
    missing = [i for i, v in enumerate(out) if v is None]
    if missing:
        raise RuntimeError(f"systems {missing[:8]} were solved by no rank")
    return out


def batched_checksum(results):
    """Checksum of checksums of the batched velocities: the float64 sum of
    every (system, right-hand side)'s per-component sums, in system order."""
    return float(sum(np.asarray(v, np.float64).sum() for per_sys in results for v in per_sys))


def measure_batched(args, rank, world, local_rank):
    import torch
    from fixtures import nonoverlapping_uniform
    ffcm = _load_product()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    b = BATCH
    systems_all = batched_systems()
    owner = shard_systems(systems_all, world)
    mine = [i for i in range(len(systems_all)) if owner[i] == rank]
    systems = [systems_all[i] for i in mine]
    rng = np.random.default_rng(b["seed"] + 1)
    Ys = [nonoverlapping_uniform(s["N"], s["L"][0], b["seed"] + 10 + i).astype(np.float32)
          for i, s in zip(mine, systems)]
    Fs = [[rng.standard_normal((s["N"], 3)).astype(np.float32) for _ in range(b["nrhs"])]
          for s in systems]
    common = dict(kernel_widths_ratio=b["ratio"], M_G=b["M_G"], viscosity=b["mu"])
    batch = ffcm.FFCMBatch(np.float32, systems=systems, nrhs=b["nrhs"], device=local_rank, **common)
    Yf, Ff = batch.pack(Ys, Fs)
    Yd, Fd = torch.from_numpy(Yf).to(dev), torch.from_numpy(Ff).to(dev)
    Vd = torch.empty_like(Fd)
    stream = torch.cuda.current_stream(dev)

    def barrier():
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
            torch.cuda.synchronize(dev)

    def timed(fn, steps):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        barrier()
        return e0.elapsed_time(e1) / steps

    for _ in range(args.warmup):
        batch.mobility(Vd, Yd, Fd)
    with ClockSampler(local_rank) as clk:
        ms_batch = timed(lambda: batch.mobility(Vd, Yd, Fd), args.steps)
    # the same solves through the plain single-system path, called sequentially
    cfgs = [ffcm.FFCMConfig(np.float32, L=s["L"], R_c=s["R_c"], N=s["N"],
                            num_grid_points=s["num_grid_points"], device=local_rank, **common)
            for s in systems]
    views = []
    for i, s in enumerate(systems):
        y = Yd[batch.yoff[i]: batch.yoff[i] + s["N"]]
        for r in range(b["nrhs"]):
            o = batch.fvoff[i] + r * s["N"]
            views.append((cfgs[i], y, Fd[o: o + s["N"]], Vd[o: o + s["N"]]))

    def plain_loop():
        for cfg, y, f, v in views:
            ffcm.mobility(v, cfg, y, f)

    plain_loop()
    ms_plain = timed(plain_loop, max(1, args.steps // 4))
    # end to end with pinned host buffers
    Yh = torch.from_numpy(Yf).pin_memory()
    Fh = torch.from_numpy(Ff).pin_memory()
    Vh = torch.empty_like(Fh).pin_memory()
    batch.mobility(Vh, Yh, Fh, stream=stream)
    ms_e2e = timed(lambda: batch.mobility(Vh, Yh, Fh, stream=stream), args.steps)
    if dist is not None:
        t = torch.tensor([ms_batch, ms_plain, ms_e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_batch, ms_plain, ms_e2e = (float(x) for x in t)
    # outside the timed region: every rank's velocities to rank 0, which
    # reports a checksum of the whole batch (the same on any rank count)
    batch.mobility(Vh, Yh, Fh, stream=stream)
    torch.cuda.synchronize(dev)
    per_sys = [[np.asarray(v, np.float64).sum(axis=0) for v in rhs] for rhs in batch.unpack(Vh.numpy())]
    allres = gather_system_results(mine, per_sys, len(systems_all), dist, rank)
    line = None
    if rank == 0:
        solves = b["nsys"] * b["nrhs"]
        grids = sorted(set(s["num_grid_points"][0] for s in systems_all))
        line = {
            "metric": f"solves/s, batched form ({b['nsys']} systems x {b['nrhs']} right-hand sides)",
            "value": solves / (ms_batch / 1e3), "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_batch,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "batched FFCM mobility: 64 suspensions, N log-uniform in [2000, "
                                   "64000], 10% volume fraction, grids " + "/".join(f"{g}^3" for g in grids)
                                   + ", 16 right-hand sides each, M_G=8, R_c=3, Sigma/sigma=2",
                       "total_particles": int(sum(s["N"] for s in systems_all)),
                       "parallelism": "systems sharded across ranks" if world > 1 else "single"},
            "plain_looped": {"value": solves / (ms_plain / 1e3), "unit": "solves/s", "ms": ms_plain,
                             "how": "ffcm_mobility per (system, right-hand side), device arrays, "
                                    "one stream"},
            "speedup_vs_plain_looped": ms_plain / ms_batch,
            "roofline": batched_roofline(systems_all, b["nrhs"], ms_batch * world),
            "e2e": {"value": solves / (ms_e2e / 1e3), "unit": "solves/s", "ms_per_step": ms_e2e,
                    "h2d_bytes_per_step": int(Yh.numel() * 4 + Fh.numel() * 4),
                    "d2h_bytes_per_step": int(Vh.numel() * 4)},
            "clocks": clk.summary(),
            "gpu_launches": int(batch.kernels_per_call * args.steps),
            "result_checksum": batched_checksum(allres),
        }
    batch.close()
    for c in cfgs:
        c.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return line if rank == 0 else None


ADJ = dict(L=161.0, N=100_000, M=256, M_G=8, R_c=3.0, ratio=2.0, mu=1.0, perturb=0.05,
           seed=2024 + 4)


def adjoint_kwargs():
    a = ADJ
    return dict(L=(a["L"],) * 3, R_c=a["R_c"], N=a["N"], kernel_widths_ratio=a["ratio"],
                viscosity=a["mu"], num_grid_points=(a["M"],) * 3, M_G=a["M_G"])


def adjoint_config():
    a = ADJ
    return {"workload": f"adjoint FFCM: J = 0.5 |V(Y, F) - V_t|^2 with dJ/dY and dJ/dF, N={a['N']}, "
                        f"L={a['L']}, grid {a['M']}^3, M_G={a['M_G']}, R_c={a['R_c']}, "
                        f"Sigma/sigma={a['ratio']}, V_t = V at Y + N(0, {a['perturb']}^2), Float32",
            "N": a["N"], "grid": [a["M"]] * 3, "M_G": a["M_G"],
            "l2": "working set ~1 GB (spectrum + u and psi grids) >> 126 MB L2; no flush needed"}


def adjoint_inputs():
    from fixtures import nonoverlapping_uniform
    a = ADJ
    Y = nonoverlapping_uniform(a["N"], a["L"], a["seed"])
    rng = np.random.default_rng(a["seed"])
    F = rng.standard_normal((a["N"], 3))
    Yp = Y + rng.normal(0.0, a["perturb"], Y.shape)
    return Y.astype(np.float32), F.astype(np.float32), Yp.astype(np.float32)


def adjoint_bytes(T_bytes=4):
    """Compulsory HBM traffic per stage of the pullback (see algorithmic_bytes)."""
    a = ADJ
    N, M = a["N"], a["M"]
    grid = 3 * M ** 3 * T_bytes
    spec = 3 * (M // 2 + 1) * M * M * 2 * T_bytes
    return {"cell_list": 12 * N + 16 * N + 4 * N,
            "spread": grid + 32 * N,
            "fft_y_fwd": 2 * spec, "fft_z_stokes": 2 * spec, "fft_y_inv": 2 * spec,
            "fft_x_inv": spec + grid,
            "interpolate": 2 * grid + 3 * 16 * N + 4 * N + 24 * N,
            "correct": 3 * 16 * N + 4 * N + 2 * 2 * 12 * N}


def measure_adjoint(args, rank, world, local_rank):
    import torch
    ffcm = _load_product()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    Y, F, Yp = adjoint_inputs()
    N = Y.shape[0]
    cfg = ffcm.FFCMConfig(np.float32, device=local_rank, **adjoint_kwargs())
    Yd, Fd = torch.from_numpy(Y).to(dev), torch.from_numpy(F).to(dev)
    Vt = torch.empty_like(Yd)
    ffcm.mobility(Vt, cfg, torch.from_numpy(Yp).to(dev), Fd)
    V, dY, dF = (torch.empty_like(Yd) for _ in range(3))
    stream = torch.cuda.current_stream(dev)

    def barrier():
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
            torch.cuda.synchronize(dev)

    def timed(fn, steps):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        barrier()
        return e0.elapsed_time(e1) / steps

    def grad_step():
        ffcm.objective_gradient(cfg, Yd, Fd, Vt, V=V, dY=dY, dF=dF)

    for _ in range(args.warmup):
        grad_step()
    launches0 = cfg.launch_count()
    with ClockSampler(local_rank) as clk:
        ms_grad = timed(grad_step, args.steps)
    launches = cfg.launch_count() - launches0
    ms_fwd = timed(lambda: ffcm.mobility(V, cfg, Yd, Fd), args.steps)
    ffcm.mobility_checkpoint(V, cfg, Yd, Fd)
    ms_ckpt = timed(lambda: ffcm.mobility_checkpoint(V, cfg, Yd, Fd), args.steps)
    lam = (V - Vt).contiguous()
    ms_pull = timed(lambda: ffcm.adjoint(dY, dF, cfg, lam), args.steps)
    cfg.profile_begin()
    for _ in range(args.steps):
        ffcm.adjoint(dY, dF, cfg, lam)
    torch.cuda.synchronize(dev)
    stages = cfg.profile_end()
    # end to end: host arrays in, V, dJ/dY, dJ/dF and J out, every step
    Yh, Fh, Th = (torch.from_numpy(a).pin_memory() for a in (Y, F, Vt.cpu().numpy()))
    Vh, dYh, dFh = (torch.empty_like(Yh).pin_memory() for _ in range(3))
    ffcm.objective_gradient(cfg, Yh, Fh, Th, V=Vh, dY=dYh, dF=dFh, stream=stream)
    ms_e2e = timed(lambda: ffcm.objective_gradient(cfg, Yh, Fh, Th, V=Vh, dY=dYh, dF=dFh, stream=stream),
                   args.steps)
    if dist is not None:
        t = torch.tensor([ms_grad, ms_fwd, ms_pull, ms_ckpt, ms_e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_grad, ms_fwd, ms_pull, ms_ckpt, ms_e2e = (float(x) for x in t)
    line = None
    if rank == 0:
        per = adjoint_bytes()
        peak, peak_kind = measured_peak_hbm()
        stage_ms = {k: v[0] / max(v[1], 1) for k, v in stages.items() if v[1] > 0}
        ks = [k for k in per if k in stage_ms]
        dom = max(ks, key=lambda k: stage_ms[k])
        achieved = per[dom] / (stage_ms[dom] / 1e3) / 1e9
        cpu = None
        if not args.skip_cpu_baseline:
            sec = cpu_adjoint_run(Y, F, Vt.cpu().numpy(), os.cpu_count() or 1)
            cpu = {"value": N / sec, "unit": "particles/s", "cores": os.cpu_count() or 1, "kind": "port",
                   "sample": "one objective-gradient evaluation of the workload by the C/pocketfft "
                             "oracle (forward, residual, pullback)"}
        line = {
            "metric": "particles/s per gradient evaluation (J, dJ/dY, dJ/dF; N=100k, 256^3, Float32)",
            "value": world * N / (ms_grad / 1e3), "unit": "particles/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_grad,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {**adjoint_config(), "parallelism": "replicas" if world > 1 else "single"},
            "forward_ms": ms_fwd, "checkpointed_forward_ms": ms_ckpt, "pullback_ms": ms_pull,
            "pullback_cost_vs_forward": ms_pull / ms_fwd,
            "gradient_step_cost_vs_forward": ms_grad / ms_fwd,
            "e2e": {"value": world * N / (ms_e2e / 1e3), "unit": "particles/s", "ms_per_step": ms_e2e,
                    "h2d_bytes_per_step": int(3 * Yh.numel() * 4),
                    "d2h_bytes_per_step": int(3 * Yh.numel() * 4 + 8)},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "traffic": None,
                         "algorithmic_bytes_per_launch": per[dom]},
            "pullback_stage_ms": {k: round(v, 4) for k, v in stage_ms.items()},
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
        }
    cfg.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return line if rank == 0 else None


CLUS = dict(L=300.0, N=2_000_000, M=1024, M_G=8, R_c=3.0, ratio=2.0, mu=1.0, nclusters=2000, nrhs=8,
            perturb=0.05, seed=2024 + 5)


def clustered_kwargs():
    c = CLUS
    return dict(L=(c["L"],) * 3, R_c=c["R_c"], N=c["N"], kernel_widths_ratio=c["ratio"],
                viscosity=c["mu"], num_grid_points=(c["M"],) * 3, M_G=c["M_G"])


def measure_clustered(args, rank, world, local_rank):
    """2,000,000 particles in 2,000 Gaussian clusters (L = 300, 1024^3): a plain
    solve, the fixed-position operator over 8 right-hand sides, and the
    objective gradient per right-hand side."""
    import ctypes
    import torch
    from fixtures import clustered_gaussian
    ffcm = _load_product()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    c = CLUS
    Y = clustered_gaussian(c["N"], c["L"], c["nclusters"], c["seed"]).astype(np.float32)
    rng = np.random.default_rng(c["seed"])
    Fs = [rng.standard_normal((c["N"], 3)).astype(np.float32) for _ in range(c["nrhs"])]
    Yp = (Y + rng.normal(0.0, c["perturb"], Y.shape)).astype(np.float32) % np.float32(c["L"])
    cfg = ffcm.FFCMConfig(np.float32, device=local_rank, **clustered_kwargs())
    Yd = torch.from_numpy(Y).to(dev)
    Fd = [torch.from_numpy(f).to(dev) for f in Fs]
    V = torch.empty_like(Yd)
    Vts = []
    for f in Fd:
        vt = torch.empty_like(Yd)
        ffcm.mobility(vt, cfg, torch.from_numpy(Yp).to(dev), f)
        Vts.append(vt)
    stream = torch.cuda.current_stream(dev)
    sh = ctypes.c_void_p(stream.cuda_stream or 1)
    lib = ffcm.L_.load()

    def barrier():
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
            torch.cuda.synchronize(dev)

    def timed(fn, steps):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        barrier()
        return e0.elapsed_time(e1) / steps

    def plain():
        ffcm.mobility(V, cfg, Yd, Fd[0])

    for _ in range(args.warmup):
        plain()
    launches0 = cfg.launch_count()
    with ClockSampler(local_rank) as clk:
        ms_plain = timed(plain, args.steps)
    launches = cfg.launch_count() - launches0
    cfg.profile_begin()
    plain()
    torch.cuda.synchronize(dev)
    stages = cfg.profile_end()
    tuning = cfg.tuning()

    def apply_all():
        assert lib.ffcm_set_positions(cfg.handle, ctypes.c_void_p(Yd.data_ptr()), 1, sh) == 0
        for f in Fd:
            assert lib.ffcm_mobility_apply(cfg.handle, ctypes.c_void_p(V.data_ptr()),
                                           ctypes.c_void_p(f.data_ptr()), 1, sh) == 0

    apply_all()
    ms_apply = timed(apply_all, max(1, args.steps // 4))
    dY, dF = torch.empty_like(Yd), torch.empty_like(Yd)

    def gradients():
        for f, vt in zip(Fd, Vts):
            ffcm.objective_gradient(cfg, Yd, f, vt, V=V, dY=dY, dF=dF)

    gradients()
    ms_grad = timed(gradients, max(1, args.steps // 4))
    # end to end: host arrays through the public API (one solve)
    Yh, Fh = torch.from_numpy(Y).pin_memory(), torch.from_numpy(Fs[0]).pin_memory()
    Vh = torch.empty_like(Yh).pin_memory()
    ffcm.mobility(Vh, cfg, Yh, Fh, stream=stream)
    ms_e2e = timed(lambda: ffcm.mobility(Vh, cfg, Yh, Fh, stream=stream), args.steps)
    if dist is not None:
        t = torch.tensor([ms_plain, ms_apply, ms_grad, ms_e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_plain, ms_apply, ms_grad, ms_e2e = (float(x) for x in t)
    line = None
    if rank == 0:
        N = c["N"]
        stage_ms = {k: round(v[0] / max(v[1], 1), 4) for k, v in stages.items() if v[1] > 0}
        line = {
            "metric": "particles/s per mobility solve (clustered, N=2M, 1024^3, Float32)",
            "value": world * N / (ms_plain / 1e3), "unit": "particles/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_plain,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: 2,000 Gaussian clusters, centres uniform, std log-normal(ln 3, 0.5); "
                    "overlap allowed (a non-overlap test jams at 31%)",
            "config": {"workload": "clustered FFCM mobility: N=2000000, L=300, grid 1024^3, M_G=8, R_c=3, "
                                   "Sigma/sigma=2, 8 right-hand sides, Float32",
                       "N": N, "grid": [1024] * 3,
                       "l2": "spectrum 12.9 GB >> 126 MB L2; no flush needed",
                       "parallelism": "replicas" if world > 1 else "single"},
            "roofline": stage_roofline(stage_ms, ((c["L"],) * 3, N, (c["M"],) * 3)),
            "fixed_position_operator_ms_per_rhs": ms_apply / c["nrhs"],
            "gradient_ms_per_rhs": ms_grad / c["nrhs"],
            "stage_ms": stage_ms,
            "tuning": tuning,
            "e2e": {"value": world * N / (ms_e2e / 1e3), "unit": "particles/s", "ms_per_step": ms_e2e,
                    "h2d_bytes_per_step": int(Yh.numel() * 8), "d2h_bytes_per_step": int(Vh.numel() * 4)},
            "cpu_baseline": None,
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
        }
    cfg.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return line if rank == 0 else None


def _print_line(line):
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


def run_batched(args, rank, world, local_rank):
    return _print_line(measure_batched(args, rank, world, local_rank))


def run_adjoint(args, rank, world, local_rank):
    return _print_line(measure_adjoint(args, rank, world, local_rank))


def run_clustered(args, rank, world, local_rank):
    return _print_line(measure_clustered(args, rank, world, local_rank))


RES_METRIC = ("particles/s per CG iteration of the resistance solve M(Y) F = V "
              "(N=500k, 512^3, Float32, to |r| <= sqrt(eps) |V|)")


def resistance_config():
    c = workload_config()
    c["workload"] = ("resistance solve M(Y) F = V by conjugate gradients on the mobility operator "
                     "(IterativeSolvers cg stopping rule, reltol = sqrt(eps(Float32)), F0 = 0); "
                     + c["workload"].replace("plain FFCM mobility, ", ""))
    return c


def resistance_inputs():
    Y, _ = make_inputs()
    V = np.random.default_rng(WORK["seed"] + 7).standard_normal(Y.shape).astype(np.float32)
    return Y, V


def run_resistance(args, rank, world, local_rank):
    line, dist = measure_resistance(args, rank, world, local_rank)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def measure_resistance(args, rank, world, local_rank):
    """The resistance solve's line (rank 0; None elsewhere) and the process
    group (None on one GPU)."""
    import torch
    ffcm = _load_product()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    Y, V = resistance_inputs()
    N = Y.shape[0]
    cfg = ffcm.FFCMConfig(np.float32, device=local_rank, **config_kwargs())
    Yd, Vd = torch.from_numpy(Y).to(dev), torch.from_numpy(V).to(dev)
    Fd = torch.empty_like(Yd)
    stream = torch.cuda.current_stream(dev)
    op = ffcm.FFCMMobility(cfg, Yd)

    def barrier():
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
            torch.cuda.synchronize(dev)

    def timed(fn, steps):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        barrier()
        return e0.elapsed_time(e1) / steps

    hist = []

    def solve():
        # positions fixed (wrap, hash, sort) and the whole CG loop: one resistance solve
        op._set_positions()
        hist.append(ffcm.cg(op, Vd, out=Fd, log=True)[1])

    for _ in range(args.warmup):
        solve()
    launches0 = cfg.launch_count()
    hist.clear()
    with ClockSampler(local_rank) as clk:
        ms = timed(solve, args.steps)
    launches = cfg.launch_count() - launches0
    # the operator sums slab shares with atomics, so the F32 iteration count
    # may differ by one between solves: the metric counts the iterations run
    iters = sum(h.iters for h in hist) / len(hist)
    # one operator application alone (the iteration's dominant part)
    lib = ffcm.L_.load()
    sh = ffcm._stream_handle(stream)
    W = torch.empty_like(Yd)
    ms_apply = timed(lambda: lib.ffcm_mobility_apply(cfg.handle, W.data_ptr(), Fd.data_ptr(), 1, sh), args.steps)
    cfg.profile_begin()
    lib.ffcm_mobility_apply(cfg.handle, W.data_ptr(), Fd.data_ptr(), 1, sh)
    torch.cuda.synchronize(dev)
    stages = cfg.profile_end()
    # end to end: host Y and V in, F out, every step
    Yh, Vh = torch.from_numpy(Y).pin_memory(), torch.from_numpy(V).pin_memory()
    Fh = torch.empty_like(Yh).pin_memory()

    def solve_host():
        o = ffcm.FFCMMobility(cfg, Yh)
        ffcm.cg(o, Vh, out=Fh)

    solve_host()
    ms_e2e = timed(solve_host, args.steps)
    if dist is not None:
        t = torch.tensor([ms, ms_apply, ms_e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_apply, ms_e2e = (float(x) for x in t)
    if rank == 0:
        per, solve_bytes = algorithmic_bytes()
        peak, peak_kind = measured_peak_hbm()
        stage_ms = {k: v[0] / max(v[1], 1) for k, v in stages.items() if v[1] > 0}
        ks = [k for k in per if k in stage_ms]
        dom = max(ks, key=lambda k: stage_ms[k])
        achieved = per[dom] / (stage_ms[dom] / 1e3) / 1e9
        # per iteration: one application without the cell list, plus the CG
        # vector kernels (direction: 2 reads 1 write; alpha: 2 reads; update: 4 reads 2 writes)
        it_bytes = solve_bytes - per["cell_list"] + 11 * 3 * N * 4
        ms_iter = ms / max(iters, 1)
        cpu = None
        if not args.skip_cpu_baseline:
            import ffcm_oracle as O
            threads = os.cpu_count() or 1
            ocfg = O.OracleConfig(np.float32, **config_kwargs(), fft_threads=threads)
            t0 = time.perf_counter()
            O.cg(ocfg, Y, V, maxiter=1)
            sec = time.perf_counter() - t0
            cpu = {"value": N / sec, "unit": "particles/s", "cores": threads, "kind": "port",
                   "sample": "one CG iteration (one operator application + vector updates) of the "
                             "workload by the C/pocketfft oracle"}
        line = {
            "metric": RES_METRIC, "value": world * N * iters / (ms / 1e3), "unit": "particles/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {**resistance_config(), "parallelism": "replicas" if world > 1 else "single"},
            "iterations": iters, "iterations_per_solve": [h.iters for h in hist],
            "status": sorted({h.status for h in hist}),
            "resnorm_rel": hist[-1].resnorm / float(np.linalg.norm(V.astype(np.float64))),
            "solves_per_s": world * 1e3 / ms, "ms_per_iteration": ms_iter, "apply_ms": ms_apply,
            "cg_overhead_per_iteration_ms": ms_iter - ms_apply,
            "e2e": {"value": world * N * iters / (ms_e2e / 1e3), "unit": "particles/s", "ms_per_step": ms_e2e,
                    "h2d_bytes_per_step": int(Yh.numel() * 4 + Vh.numel() * 4),
                    "d2h_bytes_per_step": int(Fh.numel() * 4)},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "traffic": ncu_traffic(dom),
                         "algorithmic_bytes_per_launch": per[dom]},
            "iteration_roofline": {"algorithmic_bytes": it_bytes,
                                   "achieved_GBs": it_bytes / (ms_iter / 1e3) / 1e9,
                                   "frac": it_bytes / (ms_iter / 1e3) / 1e9 / peak},
            "apply_stage_ms": {k: round(v, 4) for k, v in stage_ms.items()},
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
        }
    else:
        line = None
    cfg.close()
    return line, dist


SPLIT_METRIC = "particles/s per mobility solve of one system split over the GPUs by z slabs (N=500k, 512^3, Float32)"


def run_split(args, rank, world, local_rank):
    """The plain workload as ONE system over all ranks (ffcm_dist_*): each
    rank spreads, transforms along y and interpolates its own z planes and
    runs the z pass on its own kx columns; two spectrum transposes
    (all_to_all over NCCL) and one sum of the interpolation shares
    (all_reduce, 3N values) per solve. Strong scaling: the system is fixed."""
    import torch
    ffcm = _load_product()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
        exchange = ffcm.TorchExchange()
    else:
        exchange = ffcm.LocalExchange()
    Y, F = make_inputs()
    N = Y.shape[0]
    cfg = ffcm.DistributedConfig(np.float32, rank=rank, nranks=world, device=local_rank, **config_kwargs())
    Yd, Fd = torch.from_numpy(Y).to(dev), torch.from_numpy(F).to(dev)
    Vd = torch.empty_like(Yd)
    stream = torch.cuda.current_stream(dev)

    def barrier():
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
            torch.cuda.synchronize(dev)

    def timed(fn, steps):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        barrier()
        return e0.elapsed_time(e1) / steps

    def step():
        cfg.mobility(Vd, Yd, Fd, exchange)

    for _ in range(args.warmup):
        step()
    launches0 = cfg.launch_count()
    with ClockSampler(local_rank) as clk:
        ms = timed(step, args.steps)
    launches = cfg.launch_count() - launches0
    cfg.profile_begin()
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize(dev)
    stages = cfg.profile_end()
    # the exchange alone (two transposes and the sum)
    ms_exchange = timed(lambda: (exchange.all_to_all(cfg.recv, cfg.send), exchange.all_to_all(cfg.recv, cfg.send),
                                 exchange.all_reduce(cfg.partial)), args.steps)
    # end to end: pinned host Y, F in and V out through the same entry points
    Yh, Fh = torch.from_numpy(Y).pin_memory(), torch.from_numpy(F).pin_memory()
    Vh = torch.empty_like(Yh).pin_memory()
    cfg.mobility(Vh, Yh, Fh, exchange)
    ms_e2e = timed(lambda: cfg.mobility(Vh, Yh, Fh, exchange), args.steps)
    # every rank holds all N velocities: compare with the single-system solve
    Vs = Vd.cpu().numpy()
    if dist is not None:
        t = torch.tensor([ms, ms_e2e, ms_exchange], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_e2e, ms_exchange = (float(x) for x in t)
    line = None
    if rank == 0:
        one = ffcm.FFCMConfig(np.float32, device=local_rank, **config_kwargs())
        V1 = np.empty_like(Y)
        ffcm.mobility(V1, one, Y, F)
        one.close()
        peak, peak_kind = measured_peak_hbm()
        stage_ms = {k: v[0] / max(v[1], 1) for k, v in stages.items() if v[1] > 0}
        per, solve_bytes = algorithmic_bytes()
        # this rank's share of the grid traffic plus its transpose copies
        mz = cfg.ranges[1] - cfg.ranges[0]
        share = mz / work_geometry()[2][2]
        line = {
            "metric": SPLIT_METRIC, "value": N / (ms / 1e3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {**workload_config(), "parallelism": f"z-slab decomposition over {world} rank(s)",
                       "ranges_rank0": list(cfg.ranges)},
            "e2e": {"value": N / (ms_e2e / 1e3), "unit": UNIT, "ms_per_step": ms_e2e,
                    "h2d_bytes_per_step": int(Yh.numel() * 4 + Fh.numel() * 4),
                    "d2h_bytes_per_step": int(Vh.numel() * 4)},
            "exchange_ms": ms_exchange,
            "exchange_bytes_per_rank": int(2 * cfg.send.numel() * 4 + cfg.partial.numel() * 4),
            "stage_ms": {k: round(v, 4) for k, v in stage_ms.items()},
            "grid_share": share,
            "rel_l2_vs_single_gpu": float(np.linalg.norm(Vs - V1) / np.linalg.norm(V1)),
            "solve_roofline": {"algorithmic_bytes_per_rank": solve_bytes * share,
                               "achieved_GBs": solve_bytes * share / (ms / 1e3) / 1e9,
                               "peak": peak, "peak_source": peak_kind},
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
        }
    cfg.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def cpu_adjoint_run(Y, F, Vt, threads):
    import ffcm_oracle as O
    cfg = O.OracleConfig(np.float32, **adjoint_kwargs(), fft_threads=threads)
    t0 = time.perf_counter()
    O.objective_gradient(cfg, Y, F, Vt)
    return time.perf_counter() - t0


def _load_product():
    import importlib.util
    if "ffcm_b200" in sys.modules:
        return sys.modules["ffcm_b200"]
    pkg = ROOT / "ffcm.jl_b200"
    spec = importlib.util.spec_from_file_location("ffcm_b200", pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    ffcm = importlib.util.module_from_spec(spec)
    sys.modules["ffcm_b200"] = ffcm
    spec.loader.exec_module(ffcm)
    return ffcm


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--skip-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="plain workload only: no batched/adjoint/clustered/resistance sub-objects")
    ap.add_argument("--workload", choices=["plain", "batched", "adjoint", "clustered", "resistance", "split"], default="plain")
    ap.add_argument("--grid", default=None,
                    help="Mx,My,Mz: smaller case at the same spacing and density (profiling)")
    args = ap.parse_args()
    global GRID
    if args.grid:
        GRID = tuple(int(x) for x in args.grid.split(","))
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        # one process per GPU: start them through torch.distributed.run
        import socket
        import subprocess
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
               "--master-addr=127.0.0.1", f"--master-port={port}", str(Path(__file__).resolve())] + sys.argv[1:]
        return subprocess.call(cmd)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if world != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}; launch one process per GPU",
              file=sys.stderr)
        return 2
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "batched":
        return run_batched(args, rank, world, local_rank)
    if args.workload == "adjoint":
        return run_adjoint(args, rank, world, local_rank)
    if args.workload == "clustered":
        return run_clustered(args, rank, world, local_rank)
    if args.workload == "resistance":
        return run_resistance(args, rank, world, local_rank)
    if args.workload == "split":
        return run_split(args, rank, world, local_rank)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
