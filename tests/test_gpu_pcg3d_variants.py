"""3D pressure PCG in MIXED precision: the single-reduction variant (one
TMA-staged stencil launch per iteration, selected by FLURSYS_PCG_CG1=1)
against the FP64 oracle and against the standard two-launch PCG (the
default), in each of its launch forms."""
import numpy as np
import pytest

from flursys_b200 import _abi
from flursys_b200.solver import _Handle

from .test_gpu_cavity3d import FIELDS, MIXED_TOL, cfg3d

pytestmark = pytest.mark.gpu


def _run(oracle, shape, steps, monkeypatch, env, rtol=1e-8, max_iters=20000):
    env = dict(env)
    env.setdefault("FLURSYS_PCG_CG1", "1")
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    cfg = cfg3d(oracle, *shape, rtol=rtol, precision=_abi.PRECISION_MIXED)
    cfg.pressure_max_iters = max_iters
    gpu = _Handle(cfg)
    reps = [gpu.step(1) for _ in range(steps)]
    fields = {fid: gpu.download(fid) for fid, _ in FIELDS}
    for k in env:
        monkeypatch.delenv(k)
    return reps, fields


def _vel_rel(a, b):
    """||(u, v, w)_a - (u, v, w)_b||_2 / ||(u, v, w)_b||_2."""
    num = sum(float(np.sum((a[fid] - b[fid]) ** 2)) for fid, _ in FIELDS[:3])
    den = sum(float(np.sum(b[fid] ** 2)) for fid, _ in FIELDS[:3])
    return (num / den) ** 0.5


@pytest.mark.parametrize("shape,env", [
    ((32, 32, 32), {}),
    ((36, 26, 22), {}),                                    # partial tiles in x, y and z
    ((20, 40, 9), {"FLURSYS_CG1_TZ": "4"}),                # 4-plane tiles
    ((32, 32, 32), {"FLURSYS_PCG_VARIANT": "host"}),       # host-driven launches
    ((30, 26, 22), {}),                                    # nx % 4 != 0: the two-launch form
])
def test_single_reduction_pcg_against_fp64_oracle(oracle, monkeypatch, shape, env):
    cfg64 = cfg3d(oracle, *shape, rtol=1e-8)
    ref = oracle.OracleSolver(cfg64)
    steps = 5
    for _ in range(steps):
        ref.step(1)
    reps, fields = _run(oracle, shape, steps, monkeypatch, env)
    for rep in reps:
        assert rep.pressure_status == _abi.LINEAR_CONVERGED
        assert rep.pressure_true_relative_residual <= 1.0e-8 * 1.0001
    # velocity as one field: a thin z-velocity on anisotropic grids would
    # make its own relative norm noisy at a 1e-8 pressure stop
    assert _vel_rel(fields, {fid: ref.get(fid) for fid, _ in FIELDS[:3]}) <= MIXED_TOL


def test_single_reduction_iterations_track_standard_pcg(oracle, monkeypatch):
    shape = (48, 40, 32)  # > 100 iterations: two residual replacements inside each solve
    one, f1 = _run(oracle, shape, 3, monkeypatch, {})
    two, f2 = _run(oracle, shape, 3, monkeypatch, {"FLURSYS_PCG_CG1": "0", "FLURSYS_PCG_RESIDENT": "0"})
    for a, b in zip(one, two):
        assert a.pressure_status == b.pressure_status == _abi.LINEAR_CONVERGED
        assert b.pressure_iterations > 100
        assert abs(a.pressure_iterations - b.pressure_iterations) <= 2
    assert _vel_rel(f1, f2) <= MIXED_TOL


def test_single_reduction_iteration_cap(oracle, monkeypatch):
    reps, fields = _run(oracle, (32, 32, 32), 1, monkeypatch, {}, rtol=1e-12, max_iters=37)
    rep = reps[0]
    assert rep.pressure_status == _abi.LINEAR_MAX_ITERATIONS
    assert rep.pressure_iterations == 37
    assert all(np.isfinite(v).all() for v in fields.values())
