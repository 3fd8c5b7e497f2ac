"""Benchmark of the 3D lid-driven-cavity projection step on B200.

Workload (one "step" = one projection step: predictor, divergence RHS,
pressure Poisson solve, correction, diagnostics): 3D lid-driven cavity,
128^3 cells on the unit cube, lid u = 1, Re = 400, central convection,
dt = min(0.5 h/U, 0.25 h^2/(3 nu)), mixed precision (FP32 stencil/SpMV
vectors, FP64 dots, FP64 residual replacement every 50 iterations and FP64
final residual check), Jacobi-PCG to 1e-8 relative residual (L2).

Metric: cell-steps/s (cells x steps / device time). Inputs stay resident in
HBM for `value`; `e2e` runs the same steps through the public API with the
state copied host->device before and device->host after every step.

Arms:
  default            the CUDA backend (libflursys_cuda.so)
  --impl reference   the reference CPU path restated in C++ (oracle/), all
                     host threads, bounded sample of the same workload.
Extra lines on the same JSON object (rank 0): the 256^3 plain-PCG solve and
the learned-FCG solve at the same stop rule (pcg_big, fcg_big), the batched
2D cavities (batch2d), the 2D 128^2 cavity (cavity2d_128) and the steady
SIMPLE channel (simple_channel).
Multi-GPU (torchrun): replicas only — every rank advances its own cavity; no
collective is on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "pcg3d_traffic.json")
FALLBACK_HBM_GBS = 6650.0


def workload_config(n: int, precision: str):
    from flursys_b200 import _abi
    from flursys_b200.solver import LidDrivenCavity3DConfig, BackendOptions
    h = 1.0 / n
    re = 400.0
    nu = 1.0 / re
    dt = min(0.5 * h / 1.0, 0.25 * h * h / (3.0 * nu))
    cfg = LidDrivenCavity3DConfig(nx=n, ny=n, nz=n, reynolds=re, dt=dt, max_steps=500, pressure_max_iters=20000,
                                  pressure_solver="pcg",
                                  backend=BackendOptions(precision=precision, stop_rule="rel-l2", pressure_atol=0.0,
                                                         pressure_rtol=1e-8, residual_replacement_every=50))
    return cfg, cfg.to_c()


def pcg_bytes_per_launch(n_cells: int, iterations: int, precision: str, replace_every: int = 50) -> float:
    """Compulsory HBM bytes of one pressure solve (one graph launch).

    MIXED per cell: init 24 (read x, rhs; write r, dx), each iteration 40
    (operand pass: read r, d_old, write d, q — 4 B each; update pass: read
    dx, d, r, q, write dx, r), each FP64 residual replacement 44 (fold: read
    x, dx, write x; residual: read x, rhs, write r, dx), final check 16.
    F64: init 24, each iteration 80, final 16.
    """
    if precision == "mixed":
        nrep = iterations // replace_every + 1
        return float(n_cells) * (24 + 40 * iterations + 44 * nrep + 16)
    return float(n_cells) * (24 + 80 * iterations + 16)


def launches_per_step(iterations: int, precision: str, replace_every: int = 50) -> int:
    """Kernels of one 3D step: predictor (3), rhs, correction, diagnostics (2),
    and the solve graph: init, operand + update per iteration, fold + replace
    per FP64 replacement, pending fold, final check."""
    nrep = iterations // replace_every + 1 if precision == "mixed" else 0
    return 7 + 1 + 2 * iterations + 2 * nrep + (1 if precision == "mixed" else 0) + 1


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.path = os.path.join("/tmp", f"flursys_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device_index), "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for nm, val in zip(names, parts[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(nm)
        except FileNotFoundError:
            pass
        loaded = [s for s in sm if smax and s > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, value: float, device) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_reference_run(n: int, max_steps: int, budget_s: float, threads: int):
    """Times the oracle (C++ restatement of the reference CPU path) on this host."""
    from oracle import binding as ob
    ob.set_threads(threads)
    _, c = workload_config(n, "f64")
    solver = ob.OracleSolver(c)
    t0 = time.perf_counter()
    steps = 0
    its = []
    while steps < max_steps:
        rep = solver.step(1)
        steps += 1
        its.append(int(rep.pressure_iterations))
        if time.perf_counter() - t0 > budget_s:
            break
    elapsed = time.perf_counter() - t0
    return steps, elapsed, its


def run_reference(args):
    world, rank, _ = dist_setup()
    n = args.size
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    threads = os.cpu_count() or 1
    steps, elapsed, its = cpu_reference_run(n, args.steps, args.reference_budget, threads)
    value = n ** 3 * steps / elapsed
    line = {
        "impl": "reference", "metric": "3D cavity cell-steps/s", "value": value, "unit": "cell-steps/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": 0, "ms_per_step": 1000.0 * elapsed / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"3D lid-driven cavity {n}^3, Re 400, central, PCG 1e-8 rel L2",
                   "cells": n ** 3, "pressure_iterations": its},
        "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": threads, "kind": "port",
                         "sample": f"{steps} of the requested {args.steps} projection steps of the {n}^3 cavity "
                                   f"from the zero initial field (bounded at {args.reference_budget:.0f} s)"},
        "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    print(json.dumps(line))


def run_ours(args):
    import numpy as np
    import torch

    from flursys_b200 import _abi
    from flursys_b200.solver import _Handle

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.size
    precision = args.precision
    pycfg, c = workload_config(n, precision)
    c.device = local
    stream = torch.cuda.current_stream(dev)
    h = _Handle(c)
    h.set_stream(stream.cuda_stream)
    n_cells = n ** 3
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2

    for _ in range(args.warmup):
        h.step(1)
    torch.cuda.synchronize(dev)
    barrier(world)
    torch.cuda.synchronize(dev)

    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    step_ms, solve_ms, its, true_rel = [], [], [], []
    for _ in range(args.steps):
        flush.zero_()  # evict L2 between timed steps (outside the events)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rep = h.step(1)
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        solve_ms.append(rep.pressure_solve_ms)
        its.append(int(rep.pressure_iterations))
        true_rel.append(rep.pressure_true_relative_residual)
    torch.cuda.synchronize(dev)
    clocks = sampler.stop() if sampler else None
    barrier(world)
    total_ms = max_over_ranks(world, float(sum(step_ms)), dev)
    value = world * n_cells * args.steps / (total_ms / 1000.0)

    # e2e: the same steps through the public API with host-resident state.
    fields = [_abi.FIELD_U, _abi.FIELD_V, _abi.FIELD_W, _abi.FIELD_PRESSURE]
    host = {f: torch.from_numpy(h.download(f)).pin_memory() for f in fields}
    hbytes = sum(host[f].numel() * 8 for f in fields)
    torch.cuda.synchronize(dev)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for f in fields:
            h.upload(f, host[f].numpy())
        rep = h.step(1)
        for f in fields:
            h.download(f, host[f].numpy())
    torch.cuda.synchronize(dev)
    e2e_s = max_over_ranks(world, time.perf_counter() - t0, dev)
    e2e_value = world * n_cells * args.steps / e2e_s
    report_bytes = 2 * 80 + 48  # PcgResultDev + Diag3Dev read back per step
    h.close()

    if rank == 0:
        line = {
            "metric": "3D cavity cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic",
            "config": {"workload": f"3D lid-driven cavity {n}^3, Re 400, central, mixed PCG 1e-8 rel L2",
                       "cells": n_cells, "precision": precision, "l2": "flushed between timed steps (256 MiB write)",
                       "pressure_iterations": its, "pressure_solve_ms": solve_ms,
                       "true_relative_residual_max": max(true_rel), "parallelism": f"replicas{world}"},
            "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": hbytes,
                    "d2h_bytes_per_step": hbytes + report_bytes},
            "gpu_launches": sum(launches_per_step(i, precision) for i in its),
            "clocks": clocks,
        }
        line["roofline"] = roofline(n_cells, its, solve_ms, precision)
        if args.big_size and not args.no_big:
            line["pcg_big"] = big_solve(args.big_size, precision, local)
            line["fcg_big"] = fcg_solve(args.big_size, precision, local, line["pcg_big"])
        if not args.no_extra:
            line["batch2d"] = batch2d_run(local)
            line["cavity2d_128"] = cavity2d_run(local)
            line["simple_channel"] = simple_run()
        if not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            steps, elapsed, cits = cpu_reference_run(n, 3, args.cpu_budget, threads)
            line["cpu_baseline"] = {"value": n_cells * steps / elapsed, "unit": "cell-steps/s", "cores": threads,
                                    "kind": "port",
                                    "sample": f"{steps} projection step(s) of the {n}^3 cavity from the zero field, "
                                              f"FP64 oracle, PCG iterations {cits}"}
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def big_solve(n, precision, device):
    """Two steps of the n^3 cavity, plain PCG: pressure-solve ms, iterations
    and HBM roofline of the second (warm-started) solve."""
    from flursys_b200.solver import _Handle
    _, c = workload_config(n, precision)
    c.device = device
    h = _Handle(c)
    h.step(1)  # first step from the zero field; the second is timed
    rep = h.step(1)
    h.close()
    its = int(rep.pressure_iterations)
    r = roofline(n ** 3, [its], [rep.pressure_solve_ms], precision)
    return {"cells": n ** 3, "pressure_iterations": its, "pressure_solve_ms": rep.pressure_solve_ms,
            "step_ms": rep.step_ms, "true_relative_residual": rep.pressure_true_relative_residual,
            "roofline_frac": r["frac"], "achieved_gbs": r["achieved"]}


def fcg_solve(n, precision, device, pcg):
    """The same two steps with the learned-preconditioner FCG (trained weights
    shipped in flursys_b200/weights): pressure-solve ms at the same stop rule
    (FP64 ||b - A x||_2 <= 1e-8 ||b - A x0||_2), against the plain PCG."""
    import os as _os
    from flursys_b200.learned import DEFAULT_WEIGHTS
    from flursys_b200.solver import _Handle
    if not _os.path.exists(DEFAULT_WEIGHTS):
        return {"unavailable": "no trained weights file"}
    _, c = workload_config(n, precision)
    c.device = device
    c.pressure_solver = 2  # FLURSYS_PRESSURE_FCG
    c.fcg_weights_path = _os.fsencode(DEFAULT_WEIGHTS)
    h = _Handle(c)
    h.step(1)
    rep = h.step(1)
    h.close()
    out = {"cells": n ** 3, "pressure_iterations": int(rep.pressure_iterations),
           "pressure_solve_ms": rep.pressure_solve_ms, "fallback": int(rep.fcg_fallback),
           "true_relative_residual": rep.pressure_true_relative_residual,
           "iterations_ratio_pcg_over_fcg": pcg["pressure_iterations"] / max(1, int(rep.pressure_iterations)),
           "speedup_vs_pcg": pcg["pressure_solve_ms"] / rep.pressure_solve_ms}
    return out


def batch2d_run(device, instances=64, steps=5, warmup=2, seed=2024):
    """Config of the batched solver: 64 independent 2D cavities, sides drawn
    from U{64..512}, Re from U[100, 2000], adaptive dt (CFL 0.5, diffusion
    0.25), upwind, mixed precision, PCG to 1e-8 relative L2; aggregate
    cell-steps/s of whole batch steps (one graph launch each)."""
    import ctypes as C
    import numpy as np
    import torch
    from flursys_b200 import _abi
    from flursys_b200.solver import BatchedIncompressibleSolver
    lib = _abi.load()
    rng = np.random.default_rng(seed)
    sides = rng.integers(64, 513, size=instances)
    res = rng.uniform(100.0, 2000.0, size=instances)
    cfgs = []
    for n, re in zip(sides, res):
        c = _abi.CudaConfig()
        lib.flursys_cuda_default_config(2, C.byref(c))
        c.nx = c.ny = int(n)
        c.case_params.kinematic_viscosity = 1.0 / re
        c.case_params.reynolds = re
        c.adaptive = 1
        c.dt = 1e-3
        c.target_cfl, c.target_diffusion_number = 0.5, 0.25
        c.t_end = 1e9
        c.stop_rule = _abi.STOP_REL_L2
        c.pressure_atol, c.pressure_rtol = 0.0, 1e-8
        c.pressure_max_iters = 50000
        c.precision = _abi.PRECISION_MIXED
        c.residual_replacement_every = 50
        c.device = device
        cfgs.append(c)
    cells = int((sides.astype(np.int64) ** 2).sum())
    b = BatchedIncompressibleSolver(cfgs, autotune=True)
    b.advance(warmup)
    torch.cuda.synchronize(device)
    b.advance(steps)
    reps = [b.report(i) for i in range(instances)]
    ms = reps[0].step_ms
    its = [int(r.pressure_iterations) for r in reps]
    status = sorted({b.status(i) for i in range(instances)})
    tuning = b.tuning()
    b.close()
    return {"instances": instances, "cells": cells, "sides": [int(sides.min()), int(sides.max())],
            "steps": steps, "ms_per_step": ms, "cell_steps_per_s": cells / (ms / 1000.0),
            "pressure_iterations_min_max": [min(its), max(its)], "status": status, "tuning": tuning}


def simple_run(outer=3):
    """Steady SIMPLE plane channel, 2048 x 512 cells, L 8, H 1, parabolic
    inlet (peak 1), Re 200 on the mean velocity: device ms per outer
    iteration (momentum CSR + 2 BiCGSTAB, Rhie-Chow, pressure-correction
    CSR + Jacobi-PCG, corrections), the continuity RMS after each, and the
    FP64 oracle's time for one outer iteration of the 512 x 128 channel
    beside the device's. The reference's continuity stop rule (RMS of the
    integrated cell imbalance) is met after the first pressure correction,
    so a fixed number of outer iterations is timed."""
    from flursys_b200.solver import ChannelSimpleConfig, solve_simple_channel
    opts = dict(continuity_tolerance=0.0, momentum_solver=(1e-10, 1e-8, 20000), pressure_solver=(1e-10, 1e-8, 50000))
    big = solve_simple_channel(ChannelSimpleConfig(nx=2048, ny=512, max_outer_iterations=outer, **opts))
    r = big["report"]
    out = {"cells": 2048 * 512, "outer_iterations": int(r.outer_iterations),
           "ms_per_outer": r.solve_ms / max(1, r.outer_iterations),
           "pressure_pcg_iterations": int(r.pressure.iterations),
           "momentum_bicgstab_iterations": [int(r.momentum[0].iterations), int(r.momentum[1].iterations)],
           "continuity_rms": [float(x) for x in big["history"]]}
    small = ChannelSimpleConfig(nx=512, ny=128, max_outer_iterations=1, **opts)
    dev = solve_simple_channel(small)["report"]
    out["small_512x128_device_ms_per_outer"] = dev.solve_ms
    try:
        from oracle import binding as ob
        ob.load()
        ob.set_threads(1)
        t0 = time.perf_counter()
        st = ob.simple_channel(small.to_c())[0]
        out["small_512x128_oracle_ms_per_outer"] = (time.perf_counter() - t0) * 1e3 if st == 0 else None
    except Exception as exc:  # the oracle library is a test artefact; report its absence
        out["small_512x128_oracle_ms_per_outer"] = f"unavailable: {exc}"
    return out


def cavity2d_run(device, n=128, steps=1000):
    """2D cavity 128^2, Re 100, upwind, adaptive dt (CFL 0.5, diffusion 0.25),
    PCG to 1e-8 relative L2, f64, 1000 steps from the zero field:
    cell-steps/s (host-timed: the 2D handle reads its diagnostics back every
    step, as advance() returns a SolverStep)."""
    import ctypes as C
    from flursys_b200 import _abi
    from flursys_b200.solver import _Handle
    lib = _abi.load()
    c = _abi.CudaConfig()
    lib.flursys_cuda_default_config(2, C.byref(c))
    c.nx = c.ny = n
    c.case_params.reynolds = 100.0
    c.case_params.kinematic_viscosity = 0.01
    c.adaptive = 1
    c.dt = 1e-3
    c.target_cfl, c.target_diffusion_number = 0.5, 0.25
    c.t_end = 1e9
    c.max_steps = steps
    c.stop_rule = _abi.STOP_REL_L2
    c.pressure_atol, c.pressure_rtol = 0.0, 1e-8
    c.pressure_max_iters = 50000
    c.precision = _abi.PRECISION_F64
    c.device = device
    h = _Handle(c)
    h.step(3)
    t0 = time.perf_counter()
    rep = h.step(steps)
    secs = time.perf_counter() - t0
    h.close()
    return {"cells": n * n, "steps": steps, "seconds": secs, "cell_steps_per_s": n * n * steps / secs,
            "last_pressure_iterations": int(rep.pressure_iterations), "last_dt": rep.time_step}


def roofline(n_cells, its, solve_ms, precision):
    peak, peak_src = FALLBACK_HBM_GBS, "fallback"
    try:
        peak = float(json.load(open(PEAKS_FILE))["hbm_gbs"])
        peak_src = "measured"
    except Exception:
        pass
    bytes_total = sum(pcg_bytes_per_launch(n_cells, i, precision) for i in its)
    secs = sum(solve_ms) / 1000.0
    achieved = bytes_total / secs / 1e9
    traffic = None
    try:
        t = json.load(open(TRAFFIC_FILE))[precision]
        by_size = {int(k): v for k, v in t.get("by_size", {}).items()}
        n = round(n_cells ** (1.0 / 3.0))
        per_cell_it = by_size[min(by_size, key=lambda s: abs(s - n))] if by_size else t["dram_bytes_per_cell_iteration"]
        traffic = per_cell_it * n_cells * (sum(its) / len(its))
    except Exception:
        pass
    return {"bound": "hbm", "kernel": "pressure-solve graph (seq_dir_vec + seq_update per iteration)",
            "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_src,
            "algorithmic_bytes_per_launch": bytes_total / len(its), "traffic": traffic}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "f64"])
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--reference-budget", type=float, default=120.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--big-size", type=int, default=256, help="size of the extra plain-PCG solve measurement")
    ap.add_argument("--no-big", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the batched-2D and 2D-cavity sub-measurements")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
