"""Per-phase device-time split of the 3D pressure PCG (a user-facing diagnostic).

    python -m flursys_b200.profile_pcg --size 256 --precision mixed --steps 2

Prints, per step, the iterations, the solve time and the split reported by
flursys_cuda_solver_profile (stencil / pointwise / barriers / replacements).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import subprocess

from . import _abi
from .solver import BackendOptions, LidDrivenCavity3DConfig, _Handle


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--precision", default="mixed")
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--iters", type=int, default=20000, help="pressure iteration limit")
    args = ap.parse_args()
    n = args.size
    h = 1.0 / n
    nu = 1.0 / 400.0
    cfg = LidDrivenCavity3DConfig(nx=n, ny=n, nz=n, reynolds=400.0, dt=min(0.5 * h, 0.25 * h * h / (3 * nu)),
                                  pressure_max_iters=args.iters, pressure_solver="pcg",
                                  backend=BackendOptions(precision=args.precision, stop_rule="rel-l2",
                                                         pressure_rtol=1e-8))
    hd = _Handle(cfg.to_c())
    for s in range(args.steps):
        rep = hd.step(1)
        ph = (C.c_double * 4)()
        hd.lib.flursys_cuda_solver_profile(hd.h, ph, 4)
        its = max(1, rep.pressure_iterations)
        print(json.dumps({"step": s + 1, "iterations": int(rep.pressure_iterations),
                          "solve_ms": rep.pressure_solve_ms,
                          "us_per_iteration": 1000.0 * rep.pressure_solve_ms / its,
                          "phase_us_per_iteration": {k: 1000.0 * ph[i] / its for i, k in enumerate(
                              ["stencil", "pointwise", "barrier+reduce", "replacement"])}}))
    hd.close()
    try:
        q = subprocess.run(["nvidia-smi", "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active",
                            "--format=csv,noheader"], capture_output=True, text=True, timeout=10).stdout.strip()
        print(json.dumps({"clocks_after": q}))
    except Exception:
        pass


if __name__ == "__main__":
    main()
