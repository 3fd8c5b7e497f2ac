"""Fixed, deterministic drivers of the learned-FCG network, the batched 2D
solver and the SIMPLE channel, for profilers (ncu launch lists, section
captures) and quick timings.

    python -m flursys_b200.profile_paths fcgnet --size 256 --reps 2
    python -m flursys_b200.profile_paths fcg --size 256 --steps 1
    python -m flursys_b200.profile_paths batch2d --instances 64 --steps 2
    python -m flursys_b200.profile_paths simple --nx 2048 --ny 512 --outer 1

Launches per unit: fcgnet 10 kernels per application; batch2d 9 kernels per
step (one graph launch); simple 1 kernel before the loop, then 12 kernels
and 2 device copies per outer iteration.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time

import numpy as np


def run_fcgnet(size: int, reps: int) -> dict:
    import torch
    from .learned import DEFAULT_WEIGHTS, FcgNet
    net = FcgNet(path=DEFAULT_WEIGHTS)
    n = size
    r = torch.randn(n ** 3, device="cuda", dtype=torch.float32, generator=torch.Generator("cuda").manual_seed(0))
    z = torch.empty_like(r)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        net.apply(r, z, (n, n, n), 1.0 / (n * n))
    torch.cuda.synchronize()
    return {"size": n, "reps": reps, "ms_per_apply": (time.perf_counter() - t0) * 1e3 / reps}


def run_fcg(size: int, steps: int) -> dict:
    """`steps` 3D cavity steps (Re 400, central, mixed) with the learned FCG
    pressure solve to 1e-8 relative, from the zero field."""
    from .learned import DEFAULT_WEIGHTS
    from .solver import BackendOptions, LidDrivenCavity3DConfig, _Handle
    n = size
    h = 1.0 / n
    cfg = LidDrivenCavity3DConfig(nx=n, ny=n, nz=n, reynolds=400.0, dt=min(0.5 * h, 0.25 * h * h / (3 / 400.0)),
                                  pressure_solver="fcg",
                                  backend=BackendOptions(precision="mixed", stop_rule="rel-l2", pressure_rtol=1e-8,
                                                         fcg_weights_path=DEFAULT_WEIGHTS))
    hd = _Handle(cfg.to_c())
    reps = [hd.step(1) for _ in range(steps)]
    hd.close()
    return {"size": n, "steps": steps, "iterations": [int(r.pressure_iterations) for r in reps],
            "solve_ms": [r.pressure_solve_ms for r in reps]}


def run_batch2d(instances: int, steps: int, seed: int = 2024) -> dict:
    from . import _abi
    from .solver import BatchedIncompressibleSolver
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
        c.adaptive, c.dt, c.t_end = 1, 1e-3, 1e9
        c.target_cfl, c.target_diffusion_number = 0.5, 0.25
        c.stop_rule = _abi.STOP_REL_L2
        c.pressure_atol, c.pressure_rtol, c.pressure_max_iters = 0.0, 1e-8, 50000
        c.precision = _abi.PRECISION_MIXED
        cfgs.append(c)
    b = BatchedIncompressibleSolver(cfgs, autotune=False)
    b.advance(steps)
    out = {"instances": instances, "steps": steps, "ms_per_step": b.report(0).step_ms,
           "cells": int((sides.astype(np.int64) ** 2).sum())}
    b.close()
    return out


def run_simple(nx: int, ny: int, outer: int) -> dict:
    from .solver import ChannelSimpleConfig, solve_simple_channel
    cfg = ChannelSimpleConfig(nx=nx, ny=ny, max_outer_iterations=outer, continuity_tolerance=0.0,
                              momentum_solver=(1e-10, 1e-8, 20000), pressure_solver=(1e-10, 1e-8, 50000))
    r = solve_simple_channel(cfg)["report"]
    return {"nx": nx, "ny": ny, "outer": int(r.outer_iterations), "solve_ms": r.solve_ms,
            "pressure_pcg_iterations": int(r.pressure.iterations)}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    sub = ap.add_subparsers(dest="what", required=True)
    a = sub.add_parser("fcgnet")
    a.add_argument("--size", type=int, default=256)
    a.add_argument("--reps", type=int, default=2)
    f = sub.add_parser("fcg")
    f.add_argument("--size", type=int, default=256)
    f.add_argument("--steps", type=int, default=1)
    b = sub.add_parser("batch2d")
    b.add_argument("--instances", type=int, default=64)
    b.add_argument("--steps", type=int, default=2)
    s = sub.add_parser("simple")
    s.add_argument("--nx", type=int, default=2048)
    s.add_argument("--ny", type=int, default=512)
    s.add_argument("--outer", type=int, default=1)
    args = ap.parse_args(argv)
    if args.what == "fcgnet":
        out = run_fcgnet(args.size, args.reps)
    elif args.what == "fcg":
        out = run_fcg(args.size, args.steps)
    elif args.what == "batch2d":
        out = run_batch2d(args.instances, args.steps)
    else:
        out = run_simple(args.nx, args.ny, args.outer)
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
