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
                     host threads, bounded sample of the same workload; its
                     configuration is built by the oracle alone.
Extra keys on the same JSON object (rank 0): the 256^3 plain-PCG solve and
the learned-FCG solve at the same stop rule (pcg_big, fcg_big), the learned
FCG on the 128^3 workload beside the timed PCG steps (fcg_headline), the batched
2D cavities (batch2d), the 2D 128^2 cavity (cavity2d_128), the steady
SIMPLE channel (simple_channel), and `error_vs_oracle`: the error of each
workload's fields against the FP64 oracle run on the same inputs.
Multi-GPU (torchrun): replicas only — every rank advances its own cavity; no
collective is on the data path.

Single sub-measurements for profilers (one JSON line each, no oracle except
--case errors3d):
  --case pcg       the 3D pressure solve's per-phase split (--size, --steps, --iters)
  --case velocity  the 3D step's velocity kernels: steps with a 1-iteration solve
  --case fcgnet    network applications on a random residual (--size, --reps)
  --case fcg       3D cavity steps with the learned FCG (--size, --steps)
  --case batch2d   batched 2D cavity steps (--instances, --steps)
  --case simple    SIMPLE channel outer iterations (--nx, --ny, --outer)
  --case errors3d  mixed PCG and learned FCG steps from rest against the FP64
                   oracle's steps (all host threads) at --size, --steps
"""
from __future__ import annotations

import argparse
import ctypes as C
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
RE_3D = 400.0


def workload_name(n: int) -> str:
    return f"3D lid-driven cavity {n}^3, Re 400, central, PCG to 1e-8 rel L2"


def cavity3d_dt(n: int) -> float:
    h = 1.0 / n
    return min(0.5 * h / 1.0, 0.25 * h * h / (3.0 / RE_3D))


def fill_cavity3d(cfg, n: int, precision: int, solver: int) -> None:
    """Sets the workload's fields on a FlursysCudaConfig (both arms use this,
    each on a struct built by its own library)."""
    from flursys_b200 import _abi
    cfg.nx = cfg.ny = cfg.nz = n
    cp = cfg.case_params
    cp.length = cp.height = cp.depth = 1.0
    cp.density = 1.0
    cp.reference_velocity = 1.0
    cp.reynolds = RE_3D
    cp.kinematic_viscosity = 1.0 / RE_3D
    cfg.dt = cavity3d_dt(n)
    cfg.max_steps = 500
    cfg.pressure_max_iters = 20000
    cfg.pressure_solver = solver
    cfg.stop_rule = _abi.STOP_REL_L2
    cfg.precision = precision
    cfg.pressure_atol, cfg.pressure_rtol = 0.0, 1e-8
    cfg.residual_replacement_every = 50


def workload_config(n: int, precision: str, solver: str = "pcg"):
    """The workload through the public configuration API of the package."""
    from flursys_b200.solver import LidDrivenCavity3DConfig, BackendOptions
    cfg = LidDrivenCavity3DConfig(nx=n, ny=n, nz=n, reynolds=RE_3D, dt=cavity3d_dt(n), max_steps=500,
                                  pressure_max_iters=20000, pressure_solver=solver,
                                  backend=BackendOptions(precision=precision, stop_rule="rel-l2", pressure_atol=0.0,
                                                         pressure_rtol=1e-8, residual_replacement_every=50))
    if solver == "fcg":
        from flursys_b200.learned import DEFAULT_WEIGHTS
        cfg.backend.fcg_weights_path = DEFAULT_WEIGHTS
    return cfg, cfg.to_c()


def oracle_workload_config(n: int):
    """The same workload as a config built by the oracle library alone (FP64)."""
    from flursys_b200 import _abi
    from oracle import binding as ob
    cfg = ob.default_config(3)
    fill_cavity3d(cfg, n, _abi.PRECISION_F64, _abi.PRESSURE_PCG)
    return cfg


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


def launches_per_step(iterations: int, precision: str, resident: bool, replace_every: int = 50,
                      unroll: int = 8) -> int:
    """Kernels of one 3D step: predictor (3), rhs, correction, diagnostics (2),
    and the pressure solve: one cooperative launch when it runs chip-resident;
    otherwise the solve graph's init, operand + update for each iteration of
    every loop body entered (`unroll` iterations per body), fold + replace per
    FP64 replacement, pending fold and final check."""
    if resident:
        return 7 + 1
    bodies = -(-max(iterations, 1) // unroll)
    nrep = iterations // replace_every + 1 if precision == "mixed" else 0
    return 7 + 1 + 2 * bodies * unroll + 2 * nrep + (1 if precision == "mixed" else 0) + 1


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


def sm_clock_mhz() -> float | None:
    try:
        q = subprocess.run(["nvidia-smi", "--query-gpu=clocks.sm", "--format=csv,noheader,nounits", "-i", "0"],
                           capture_output=True, text=True, timeout=10).stdout.strip().splitlines()
        return float(q[0])
    except Exception:
        return None


# --------------------------------------------------------------------------
# The oracle: CPU baseline leg and checker of the fields (FP64 restatement of
# the reference CPU path; test infrastructure, never on the measured path)
# --------------------------------------------------------------------------
def cpu_reference_run(n: int, max_steps: int, budget_s: float, threads: int, warmup: int = 0):
    """Times the oracle on this host: `warmup` untimed steps, then up to
    `max_steps` timed steps within `budget_s`. Returns (steps, seconds,
    iterations, solver); the solver holds the fields after the last step."""
    from oracle import binding as ob
    ob.set_threads(threads)
    solver = ob.OracleSolver(oracle_workload_config(n))
    for _ in range(warmup):
        solver.step(1)
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
    return steps, elapsed, its, solver


def rel_l2(a, b) -> float:
    import numpy as np
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / (nb if nb > 0 else 1.0)


def rel_max(a, b) -> float:
    import numpy as np
    mb = float(np.max(np.abs(b))) if b.size else 0.0
    return float(np.max(np.abs(a - b))) / (mb if mb > 0 else 1.0)


def field_errors(gpu_get, ref_get, fields) -> dict:
    """Per-field relative L2 / max errors, plus the velocity vector's
    relative L2 over all its components."""
    import numpy as np
    out, du, nu = {}, 0.0, 0.0
    for fid, name in fields:
        a, b = gpu_get(fid), ref_get(fid)
        out[name] = {"rel_l2": rel_l2(a, b), "rel_max": rel_max(a, b)}
        if name in ("u", "v", "w"):
            du += float(np.sum((a - b) ** 2))
            nu += float(np.sum(b ** 2))
    out["velocity_rel_l2"] = (du / nu) ** 0.5 if nu > 0 else du ** 0.5
    return out


def cavity3d_errors(n: int, steps: int, ref, device) -> dict:
    """The mixed-precision PCG and the learned FCG, each run from the zero
    field for the oracle's `steps` steps on fresh handles, against the FP64
    oracle's fields (PCG to 1e-8 rel L2 in both)."""
    from flursys_b200 import _abi
    from flursys_b200.solver import _Handle
    fields = [(_abi.FIELD_U, "u"), (_abi.FIELD_V, "v"), (_abi.FIELD_W, "w"), (_abi.FIELD_PRESSURE, "p")]
    out = {}
    for key, solver in (("pcg_mixed", "pcg"), ("fcg_mixed", "fcg")):
        if solver == "fcg":
            from flursys_b200.learned import DEFAULT_WEIGHTS
            if not os.path.exists(DEFAULT_WEIGHTS):
                out[key] = {"unavailable": "no trained weights file"}
                continue
        _, c = workload_config(n, "mixed", solver)
        c.device = device
        h = _Handle(c)
        reps = [h.step(1) for _ in range(steps)]
        e = field_errors(h.download, ref.get, fields)
        e["steps"] = steps
        e["pressure_iterations"] = [int(r.pressure_iterations) for r in reps]
        e["true_relative_residual_max"] = max(r.pressure_true_relative_residual for r in reps)
        e["bound_velocity_rel_l2"] = 1e-6
        out[key] = e
        h.close()
    return out


def cavity2d_config(cfg, n: int, re: float, precision: int):
    """2D cavity n x n, upwind, adaptive dt (CFL 0.5, diffusion 0.25), PCG to
    1e-8 relative L2, on a FlursysCudaConfig built by either library."""
    from flursys_b200 import _abi
    cfg.nx = cfg.ny = int(n)
    cfg.case_params.reynolds = re
    cfg.case_params.kinematic_viscosity = 1.0 / re
    cfg.adaptive = 1
    cfg.dt = 1e-3
    cfg.target_cfl, cfg.target_diffusion_number = 0.5, 0.25
    cfg.t_end = 1e9
    cfg.stop_rule = _abi.STOP_REL_L2
    cfg.pressure_atol, cfg.pressure_rtol = 0.0, 1e-8
    cfg.pressure_max_iters = 50000
    cfg.precision = precision
    cfg.residual_replacement_every = 50
    return cfg


def cavity2d_errors(device, n=128, steps=50) -> dict:
    """The first `steps` steps of the 2D 128^2 f64 cavity against the oracle."""
    from flursys_b200 import _abi
    from flursys_b200.solver import _Handle
    from oracle import binding as ob
    lib = _abi.load()
    c = _abi.CudaConfig()
    lib.flursys_cuda_default_config(2, C.byref(c))
    cavity2d_config(c, n, 100.0, _abi.PRECISION_F64)
    c.device = device
    h = _Handle(c)
    h.step(steps)
    ref = ob.OracleSolver(cavity2d_config(ob.default_config(2), n, 100.0, _abi.PRECISION_F64))
    ref.step(steps)
    fields = [(_abi.FIELD_U, "u"), (_abi.FIELD_V, "v"), (_abi.FIELD_PRESSURE, "p")]
    out = field_errors(h.download, ref.get, fields)
    out.update({"steps": steps, "bound": 1e-10})
    h.close()
    return out


# --------------------------------------------------------------------------
# Reference arm
# --------------------------------------------------------------------------
def run_reference(args):
    world, rank, _ = dist_setup()
    n = args.size
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    threads = os.cpu_count() or 1
    steps, elapsed, its, _ = cpu_reference_run(n, args.steps, args.reference_budget, threads, warmup=args.warmup)
    value = n ** 3 * steps / elapsed
    line = {
        "impl": "reference", "metric": "3D cavity cell-steps/s", "value": value, "unit": "cell-steps/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup, "ms_per_step": 1000.0 * elapsed / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name(n), "cells": n ** 3, "precision": "f64",
                   "l2": "not applicable (host caches)", "parallelism": f"host threads {threads}"},
        "pressure_iterations": its,
        "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": threads, "kind": "port",
                         "sample": f"{steps} of the requested {args.steps} projection steps of the {n}^3 cavity "
                                   f"after {args.warmup} untimed warm-up steps from the zero initial field "
                                   f"(bounded at {args.reference_budget:.0f} s)"},
        "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    print(json.dumps(line))


# --------------------------------------------------------------------------
# Our arm
# --------------------------------------------------------------------------
def run_ours(args):
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
    resident = h.solve_kind() == _abi.SOLVE_RESIDENT
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
            "config": {"workload": workload_name(n), "cells": n_cells, "precision": precision,
                       "l2": "flushed between timed steps (256 MiB write)", "parallelism": f"replicas{world}"},
            "pressure_iterations": its, "pressure_solve_ms": solve_ms,
            "true_relative_residual_max": max(true_rel),
            "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": hbytes,
                    "d2h_bytes_per_step": hbytes + report_bytes},
            "gpu_launches": sum(launches_per_step(i, precision, resident) for i in its),
            "pressure_solve": "chip-resident cooperative PCG" if resident else "graph-driven PCG",
            "clocks": clocks,
        }
        line["roofline"] = roofline(n_cells, its, solve_ms, precision, resident)
        errors = {}
        if args.big_size and not args.no_big:
            line["pcg_big"] = big_solve(args.big_size, precision, local, args.repeats)
            line["fcg_big"] = fcg_solve(args.big_size, precision, local, line["pcg_big"], args.repeats)
            # the learned FCG on the headline workload, against the timed PCG steps above
            pcg_here = {"pressure_solve_ms_median": statistics.median(solve_ms), "pressure_iterations": its}
            line["fcg_headline"] = fcg_solve(n, precision, local, pcg_here, args.repeats)
        if not args.no_extra:
            line["batch2d"], errors["batch2d_subset_mixed"] = batch2d_run(local)
            line["cavity2d_128"] = cavity2d_run(local)
            line["simple_channel"], errors["simple_channel"] = simple_run()
            errors["cavity2d_128_f64"] = cavity2d_errors(local)
        if not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            steps, elapsed, cits, ref = cpu_reference_run(n, 3, args.cpu_budget, threads)
            line["cpu_baseline"] = {"value": n_cells * steps / elapsed, "unit": "cell-steps/s", "cores": threads,
                                    "kind": "port",
                                    "sample": f"{steps} projection step(s) of the {n}^3 cavity from the zero field, "
                                              f"FP64 oracle, PCG iterations {cits}"}
            errors[f"cavity3d_{n}"] = cavity3d_errors(n, steps, ref, local)
            errors[f"cavity3d_{n}"]["oracle_pressure_iterations"] = cits
        if errors:
            line["error_vs_oracle"] = errors
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def big_solve(n, precision, device, repeats=3):
    """Steps of the n^3 cavity with plain PCG: the first from the zero field,
    then `repeats` warm-started steps; pressure-solve ms (median), iterations
    and HBM roofline of those, with the SM clock read after them."""
    from flursys_b200.solver import _Handle
    _, c = workload_config(n, precision)
    c.device = device
    h = _Handle(c)
    h.step(1)
    reps = [h.step(1) for _ in range(repeats)]
    h.close()
    ms = [r.pressure_solve_ms for r in reps]
    its = [int(r.pressure_iterations) for r in reps]
    r = roofline(n ** 3, its, ms, precision)
    return {"cells": n ** 3, "pressure_iterations": its, "pressure_solve_ms": ms,
            "pressure_solve_ms_median": statistics.median(ms), "step_ms": [x.step_ms for x in reps],
            "true_relative_residual": max(x.pressure_true_relative_residual for x in reps),
            "roofline_frac": r["frac"], "achieved_gbs": r["achieved"], "sm_mhz_after": sm_clock_mhz()}


def fcg_solve(n, precision, device, pcg, repeats=3):
    """The same steps with the learned-preconditioner FCG (trained weights
    shipped in flursys_b200/weights): pressure-solve ms at the same stop rule
    (FP64 ||b - A x||_2 <= 1e-8 ||b - A x0||_2), against the plain PCG."""
    from flursys_b200.learned import DEFAULT_WEIGHTS
    from flursys_b200.solver import _Handle
    if not os.path.exists(DEFAULT_WEIGHTS):
        return {"unavailable": "no trained weights file"}
    _, c = workload_config(n, precision, "fcg")
    c.device = device
    h = _Handle(c)
    h.step(1)
    reps = [h.step(1) for _ in range(repeats)]
    h.close()
    ms = [r.pressure_solve_ms for r in reps]
    its = [int(r.pressure_iterations) for r in reps]
    med = statistics.median(ms)
    return {"cells": n ** 3, "pressure_iterations": its, "pressure_solve_ms": ms, "pressure_solve_ms_median": med,
            "fallback": [int(r.fcg_fallback) for r in reps],
            "true_relative_residual": max(r.pressure_true_relative_residual for r in reps),
            "iterations_ratio_pcg_over_fcg": statistics.median(pcg["pressure_iterations"]) / max(1, statistics.median(its)),
            "speedup_vs_pcg": pcg["pressure_solve_ms_median"] / med, "sm_mhz_after": sm_clock_mhz()}


def batch_configs(lib_default, instances=64, seed=2024):
    """Config of the batched solver: independent 2D cavities, sides drawn
    from U{64..512}, Re from U[100, 2000], adaptive dt (CFL 0.5, diffusion
    0.25), upwind, mixed precision, PCG to 1e-8 relative L2."""
    import numpy as np
    from flursys_b200 import _abi
    rng = np.random.default_rng(seed)
    sides = rng.integers(64, 513, size=instances)
    res = rng.uniform(100.0, 2000.0, size=instances)
    cfgs = [cavity2d_config(lib_default(), int(s), float(re), _abi.PRECISION_MIXED) for s, re in zip(sides, res)]
    return cfgs, sides, res


def batch2d_run(device, instances=64, steps=5, warmup=2, seed=2024, repeats=3, subset=4):
    """64 independent 2D cavities advanced together: aggregate cell-steps/s
    of whole batch steps (one graph launch each; median of `repeats` runs of
    `steps` steps), then a seeded subset of instances (sides <= 256) against
    the FP64 oracle run alone on the same config for the same steps."""
    import numpy as np
    import torch
    from flursys_b200 import _abi
    from flursys_b200.solver import BatchedIncompressibleSolver
    lib = _abi.load()

    def product_default():
        c = _abi.CudaConfig()
        lib.flursys_cuda_default_config(2, C.byref(c))
        c.device = device
        return c

    cfgs, sides, res = batch_configs(product_default, instances, seed)
    cells = int((sides.astype(np.int64) ** 2).sum())
    b = BatchedIncompressibleSolver(cfgs, autotune=True)
    b.advance(warmup)
    torch.cuda.synchronize(device)
    ms = []
    for _ in range(repeats):
        b.advance(steps)
        ms.append(b.report(0).step_ms)
    total_steps = warmup + steps * repeats
    reps = [b.report(i) for i in range(instances)]
    its = [int(r.pressure_iterations) for r in reps]
    status = sorted({b.status(i) for i in range(instances)})
    tuning = b.tuning()
    med = statistics.median(ms)
    out = {"instances": instances, "cells": cells, "sides": [int(sides.min()), int(sides.max())],
           "steps": steps, "repeats": repeats, "ms_per_step": ms, "ms_per_step_median": med,
           "cell_steps_per_s": cells / (med / 1000.0), "pressure_iterations_min_max": [min(its), max(its)],
           "status": status, "tuning": tuning, "sm_mhz_after": sm_clock_mhz()}
    # checker: a seeded subset against the FP64 oracle
    errs = {"steps": total_steps, "bound_velocity_rel_l2": 1e-6, "instances": {}}
    try:
        from oracle import binding as ob
        ob.set_threads(os.cpu_count() or 1)
        pick_rng = np.random.default_rng(seed + 1)
        eligible = [i for i in range(instances) if sides[i] <= 256]
        chosen = sorted(pick_rng.choice(eligible, size=min(subset, len(eligible)), replace=False).tolist())
        fields = [(_abi.FIELD_U, "u"), (_abi.FIELD_V, "v"), (_abi.FIELD_PRESSURE, "pressure")]
        for i in chosen:
            ref = ob.OracleSolver(cavity2d_config(ob.default_config(2), int(sides[i]), float(res[i]),
                                                  _abi.PRECISION_F64))
            ref.step(total_steps)
            e = field_errors(lambda fid, i=i: b.field(i, {0: "u", 1: "v", 3: "pressure"}[fid]), ref.get, fields)
            e["side"] = int(sides[i])
            e["reynolds"] = float(res[i])
            errs["instances"][str(i)] = e
    except Exception as exc:  # the oracle library is a test artefact; report its absence
        errs = {"unavailable": f"{exc}"}
    b.close()
    return out, errs


def simple_run(outer=3):
    """Steady SIMPLE plane channel, 2048 x 512 cells, L 8, H 1, parabolic
    inlet (peak 1), Re 200 on the mean velocity: device ms per outer
    iteration (momentum CSR + 2 BiCGSTAB, Rhie-Chow, pressure-correction
    CSR + Jacobi-PCG, corrections), the continuity RMS after each, and the
    FP64 oracle's time for one outer iteration of the 512 x 128 channel
    beside the device's, with the device's fields against the oracle's. The
    reference's continuity stop rule (RMS of the integrated cell imbalance)
    is met after the first pressure correction, so a fixed number of outer
    iterations is timed."""
    import numpy as np
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
    dev = solve_simple_channel(small)
    out["small_512x128_device_ms_per_outer"] = dev["report"].solve_ms
    errs = {}
    try:
        from oracle import binding as ob
        ob.load()
        ob.set_threads(1)
        t0 = time.perf_counter()
        st, u, v, p, flux, _, _ = ob.simple_channel(small.to_c())
        out["small_512x128_oracle_ms_per_outer"] = (time.perf_counter() - t0) * 1e3 if st == 0 else None
        if st == 0:
            errs["channel_512x128_1_outer"] = {
                "u": {"rel_l2": rel_l2(dev["u"], u), "rel_max": rel_max(dev["u"], u)},
                "v": {"rel_l2": rel_l2(dev["v"], v), "rel_max": rel_max(dev["v"], v)},
                "p": {"rel_l2": rel_l2(dev["p"], p), "rel_max": rel_max(dev["p"], p)},
                "face_flux": {"rel_l2": rel_l2(dev["flux"], flux), "rel_max": rel_max(dev["flux"], flux)},
                "bound": 1e-9}
    except Exception as exc:  # the oracle library is a test artefact; report its absence
        out["small_512x128_oracle_ms_per_outer"] = f"unavailable: {exc}"
    # the 2048 x 512 velocity against the analytic Poiseuille profile u = 4y(1-y)
    nx, ny = 2048, 512
    y = (np.arange(ny) + 0.5) / ny
    ua = 4.0 * y * (1.0 - y)
    ucol = big["u"].reshape(ny, nx)
    errs["channel_2048x512_vs_analytic"] = {
        "outer_iterations": int(r.outer_iterations),
        "outlet_column_rel_max": float(np.max(np.abs(ucol[:, -1] - ua)) / np.max(ua)),
        "mid_column_rel_max": float(np.max(np.abs(ucol[:, nx // 2] - ua)) / np.max(ua))}
    return out, errs


def cavity2d_run(device, n=128, steps=1000):
    """2D cavity 128^2, Re 100, upwind, adaptive dt (CFL 0.5, diffusion 0.25),
    PCG to 1e-8 relative L2, f64, 1000 steps from the zero field:
    cell-steps/s (host-timed: the 2D handle reads its diagnostics back every
    step, as advance() returns a SolverStep)."""
    from flursys_b200 import _abi
    from flursys_b200.solver import _Handle
    lib = _abi.load()
    c = _abi.CudaConfig()
    lib.flursys_cuda_default_config(2, C.byref(c))
    cavity2d_config(c, n, 100.0, _abi.PRECISION_F64)
    c.max_steps = steps
    c.device = device
    h = _Handle(c)
    h.step(3)
    t0 = time.perf_counter()
    rep = h.step(steps)
    secs = time.perf_counter() - t0
    h.close()
    # compulsory FP64 bytes per cell and step: predictor 4, RHS 3, correction
    # 5 values, and 11 per PCG iteration (the last step's count stands for all)
    its = int(rep.pressure_iterations)
    bytes_step = n * n * 8.0 * (12 + 11 * its)
    peak = FALLBACK_HBM_GBS
    try:
        peak = float(json.load(open(PEAKS_FILE))["hbm_gbs"])
    except Exception:
        pass
    hbm = bytes_step * steps / secs / 1e9
    return {"cells": n * n, "steps": steps, "seconds": secs, "cell_steps_per_s": n * n * steps / secs,
            "last_pressure_iterations": its, "last_dt": rep.time_step,
            "hbm_gbs_equivalent": hbm, "hbm_frac": hbm / peak,
            "bound": "latency: the whole state (~1.3 MB) stays on the chip"}


def roofline(n_cells, its, solve_ms, precision, resident=False):
    """HBM roofline of the pressure solve: the compulsory bytes of the
    streamed PCG (pcg_bytes_per_launch) over the event-timed solve. The
    chip-resident solve keeps its vectors in shared memory and registers,
    so for it this is the rate an HBM-streaming PCG would need to match it
    (`basis`), and `traffic` is its own measured DRAM traffic."""
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
        t = json.load(open(TRAFFIC_FILE))[("resident_" if resident else "") + precision]
        by_size = {int(k): v for k, v in t.get("by_size", {}).items()}
        n = round(n_cells ** (1.0 / 3.0))
        per_cell_it = by_size[min(by_size, key=lambda s: abs(s - n))] if by_size else t["dram_bytes_per_cell_iteration"]
        traffic = per_cell_it * n_cells * (sum(its) / len(its))
    except Exception:
        pass
    out = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
           "frac": achieved / peak, "peak_source": peak_src,
           "algorithmic_bytes_per_launch": bytes_total / len(its), "traffic": traffic}
    if resident:
        out["kernel"] = "pcg3d_res1_kernel (one cooperative launch per solve)"
        out["basis"] = ("HBM-equivalent: compulsory bytes of the streamed MIXED PCG (40 B per cell-iteration) "
                        "over the solve time; the resident kernel's own DRAM traffic is `traffic`")
    else:
        out["kernel"] = "pressure-solve graph (seq_dir_pipe + seq_update per iteration)"
    return out


# --------------------------------------------------------------------------
# Single sub-measurements (profiler drivers)
# --------------------------------------------------------------------------
def case_pcg(args) -> dict:
    """Per-phase device-time split of the 3D pressure solve, per step."""
    from flursys_b200.solver import _Handle
    _, c = workload_config(args.size, args.precision)
    c.pressure_max_iters = args.iters
    from flursys_b200 import _abi
    hd = _Handle(c)
    rows = []
    for s in range(args.steps):
        rep = hd.step(1)
        ph = (C.c_double * 6)()
        hd.lib.flursys_cuda_solver_profile(hd.h, ph, 6)
        kind = hd.solve_kind()
        names = (["halo+direction", "operator", "reduce+barrier", "update+replacement", "barrier_wait",
                  "slowest_block_work"]
                 if kind == _abi.SOLVE_RESIDENT else ["stencil", "pointwise", "barrier+reduce", "replacement"])
        its = max(1, rep.pressure_iterations)
        rows.append({"step": s + 1, "solve_kind": int(kind), "iterations": int(rep.pressure_iterations),
                     "solve_ms": rep.pressure_solve_ms, "us_per_iteration": 1000.0 * rep.pressure_solve_ms / its,
                     "phase_us_per_iteration": {k: 1000.0 * ph[i] / its for i, k in enumerate(names)}})
    hd.close()
    return {"case": "pcg", "size": args.size, "steps": rows, "sm_mhz_after": sm_clock_mhz()}


def case_velocity(args) -> dict:
    """3D steps whose pressure solve stops after one iteration, so that the
    velocity kernels (predictor, RHS, correction, diagnostics) dominate the
    launch list; step time with CUDA events."""
    import torch
    from flursys_b200.solver import _Handle
    _, c = workload_config(args.size, args.precision)
    c.pressure_max_iters = 1
    hd = _Handle(c)
    stream = torch.cuda.current_stream()
    hd.set_stream(stream.cuda_stream)
    ms = []
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        hd.step(1)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    hd.close()
    return {"case": "velocity", "size": args.size, "step_ms": ms}


def case_fcgnet(args) -> dict:
    import torch
    from flursys_b200.learned import DEFAULT_WEIGHTS, FcgNet
    net = FcgNet(path=DEFAULT_WEIGHTS)
    n = args.size
    r = torch.randn(n ** 3, device="cuda", dtype=torch.float32, generator=torch.Generator("cuda").manual_seed(0))
    z = torch.empty_like(r)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.reps):
        net.apply(r, z, (n, n, n), 1.0 / (n * n))
    torch.cuda.synchronize()
    return {"case": "fcgnet", "size": n, "reps": args.reps, "ms_per_apply": (time.perf_counter() - t0) * 1e3 / args.reps}


def case_fcg(args) -> dict:
    from flursys_b200.solver import _Handle
    _, c = workload_config(args.size, "mixed", "fcg")
    hd = _Handle(c)
    reps = [hd.step(1) for _ in range(args.steps)]
    hd.close()
    return {"case": "fcg", "size": args.size, "steps": args.steps,
            "iterations": [int(r.pressure_iterations) for r in reps],
            "solve_ms": [r.pressure_solve_ms for r in reps], "fallback": [int(r.fcg_fallback) for r in reps]}


def case_batch2d(args) -> dict:
    import numpy as np
    from flursys_b200 import _abi
    from flursys_b200.solver import BatchedIncompressibleSolver
    lib = _abi.load()

    def product_default():
        c = _abi.CudaConfig()
        lib.flursys_cuda_default_config(2, C.byref(c))
        return c

    cfgs, sides, _ = batch_configs(product_default, args.instances)
    b = BatchedIncompressibleSolver(cfgs, autotune=False)
    b.advance(args.steps)
    out = {"case": "batch2d", "instances": args.instances, "steps": args.steps, "ms_per_step": b.report(0).step_ms,
           "cells": int((sides.astype(np.int64) ** 2).sum())}
    b.close()
    return out


def case_simple(args) -> dict:
    from flursys_b200.solver import ChannelSimpleConfig, solve_simple_channel
    cfg = ChannelSimpleConfig(nx=args.nx, ny=args.ny, max_outer_iterations=args.outer, continuity_tolerance=0.0,
                              momentum_solver=(1e-10, 1e-8, 20000), pressure_solver=(1e-10, 1e-8, 50000))
    r = solve_simple_channel(cfg)["report"]
    return {"case": "simple", "nx": args.nx, "ny": args.ny, "outer": int(r.outer_iterations),
            "solve_ms": r.solve_ms, "pressure_pcg_iterations": int(r.pressure.iterations)}


def case_errors3d(args) -> dict:
    """The mixed PCG and the learned FCG against the FP64 oracle on the
    n^3 cavity, `steps` steps from rest (the oracle on all host threads)."""
    t0 = time.perf_counter()
    steps, secs, its, ref = cpu_reference_run(args.size, args.steps, 1e9, os.cpu_count() or 1)
    out = {"case": "errors3d", "size": args.size, "steps": steps, "oracle_pressure_iterations": its,
           "oracle_seconds": secs}
    out.update(cavity3d_errors(args.size, steps, ref, 0))
    out["seconds"] = time.perf_counter() - t0
    return out


CASES = {"errors3d": case_errors3d, "pcg": case_pcg, "velocity": case_velocity, "fcgnet": case_fcgnet, "fcg": case_fcg,
         "batch2d": case_batch2d, "simple": case_simple}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "f64"])
    ap.add_argument("--cpu-budget", type=float, default=30.0)
    ap.add_argument("--reference-budget", type=float, default=120.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--big-size", type=int, default=256, help="size of the extra plain-PCG / FCG solve measurement")
    ap.add_argument("--repeats", type=int, default=3, help="warm-started solves timed per big solve")
    ap.add_argument("--no-big", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the batched-2D, 2D-cavity and SIMPLE lines")
    ap.add_argument("--case", default=None, choices=sorted(CASES), help="run one sub-measurement alone")
    ap.add_argument("--iters", type=int, default=20000, help="--case pcg: pressure iteration limit")
    ap.add_argument("--reps", type=int, default=2, help="--case fcgnet: network applications")
    ap.add_argument("--instances", type=int, default=64, help="--case batch2d")
    ap.add_argument("--nx", type=int, default=2048, help="--case simple")
    ap.add_argument("--ny", type=int, default=512, help="--case simple")
    ap.add_argument("--outer", type=int, default=1, help="--case simple")
    args = ap.parse_args()
    if args.case:
        print(json.dumps(CASES[args.case](args)))
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
