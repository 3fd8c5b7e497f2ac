"""Batched 2D solvers: every instance of a batch against the FP64 oracle run
alone on the same config, plus the batch's own controls (per-instance t_end,
graph replay, autotuning) and its config checks."""
import ctypes as C

import numpy as np
import pytest

from flursys_b200 import _abi
from flursys_b200.solver import BatchedIncompressibleSolver, SolverError

from .paritylib import assert_close, rel_l2, rel_max
from .test_gpu_cavity2d import cfg2d
from .test_oracle_solver import case_cfg

PARITY_TOL = 1e-10
FIELDS = [(_abi.FIELD_U, "u"), (_abi.FIELD_V, "v"), (_abi.FIELD_PRESSURE, "pressure"),
          (_abi.FIELD_SPEED, "speed"), (_abi.FIELD_VORTICITY, "vorticity")]


def mixed_batch(oracle):
    """Uneven sizes, both convection schemes, fixed and adaptive dt, a solid
    body with an outlet and a channel."""
    cfgs = [cfg2d(oracle, 16, 16),
            cfg2d(oracle, 24, 20, convection=_abi.CONVECTION_CENTRAL),
            cfg2d(oracle, 40, 40, dt=2e-3)]
    cfgs[0].adaptive = 1
    cfgs[0].case_params.kinematic_viscosity = 1.0 / 400.0
    cfgs[2].case_params.kinematic_viscosity = 1.0 / 1000.0
    for kind, nx, ny in [(_abi.CASE_CYLINDER, 80, 32), (_abi.CASE_CHANNEL, 40, 16)]:
        c = case_cfg(oracle, kind, nx, ny)
        c.pressure_tolerance = 1e-13
        c.pressure_max_iters = 20000
        c.t_end = 100.0
        cfgs.append(c)
    return cfgs


def oracle_runs(oracle, cfgs, steps):
    out = []
    for c in cfgs:
        ref = oracle.OracleSolver(c)
        rep = ref.step(steps)
        out.append((ref, rep))
    return out


@pytest.mark.gpu
def test_batch_instances_match_oracle_f64(oracle):
    cfgs = mixed_batch(oracle)
    steps = 4
    b = BatchedIncompressibleSolver(cfgs, autotune=False)
    b.advance(steps)
    refs = oracle_runs(oracle, cfgs, steps)
    for i, (ref, a) in enumerate(refs):
        r = b.report(i)
        assert b.status(i) == _abi.OK
        assert r.iteration == a.iteration == steps
        assert abs(r.time - a.time) <= 1e-15 * max(1.0, abs(a.time))
        assert abs(r.time_step - a.time_step) <= 1e-15
        for fid, name in FIELDS:
            assert_close(b.field(i, name), ref.get(fid), PARITY_TOL, f"instance {i} {name}")
        assert abs(r.max_speed - a.max_speed) <= 1e-12
        assert abs(r.momentum_cfl - a.momentum_cfl) <= 1e-12
        if cfgs[i].case_params.kind == _abi.CASE_CYLINDER:
            assert abs(r.drag_coefficient - a.drag_coefficient) <= 1e-8 * max(1.0, abs(a.drag_coefficient))


@pytest.mark.gpu
def test_batch_mixed_precision_error_against_f64_oracle(oracle):
    # FP32 stencils / FP64 dots with the src/linear stop rule at 1e-8
    cfgs = []
    for n, re in [(32, 100.0), (48, 1000.0), (64, 2000.0)]:
        c = cfg2d(oracle, n, n, dt=1e-3)
        c.case_params.kinematic_viscosity = 1.0 / re
        c.stop_rule = _abi.STOP_REL_L2
        c.pressure_atol, c.pressure_rtol = 0.0, 1e-8
        cfgs.append(c)
    steps = 10
    refs = oracle_runs(oracle, cfgs, steps)
    mixed = []
    for c in cfgs:
        m = _abi.CudaConfig()
        C.pointer(m)[0] = c
        m.precision = _abi.PRECISION_MIXED
        m.residual_replacement_every = 50
        mixed.append(m)
    b = BatchedIncompressibleSolver(mixed, autotune=True)
    b.advance(steps)
    for i, (ref, a) in enumerate(refs):
        assert b.status(i) == _abi.OK
        for fid, name in [(_abi.FIELD_U, "u"), (_abi.FIELD_V, "v")]:
            g, o = b.field(i, name), ref.get(fid)
            assert rel_l2(g, o) < 1e-6, (i, name, rel_l2(g, o))
        r = b.report(i)
        assert r.pressure_true_relative_residual <= 1e-8 * 1.01


@pytest.mark.gpu
def test_batch_instance_stops_at_its_t_end(oracle):
    short = cfg2d(oracle, 16, 16, dt=1e-3)
    short.t_end = 2.5e-3  # two full steps and one clamped to t_end
    long_ = cfg2d(oracle, 20, 20, dt=1e-3)
    b = BatchedIncompressibleSolver([short, long_], autotune=False)
    b.advance(6)
    assert b.status(0) == _abi.ERR_REACHED_END_TIME
    r0 = b.report(0)
    assert r0.iteration == 3 and r0.reached_end_time
    assert abs(r0.time - 2.5e-3) <= 1e-15
    assert abs(r0.time_step - 0.5e-3) <= 1e-15
    assert b.status(1) == _abi.OK and b.report(1).iteration == 6
    ref = oracle.OracleSolver(short)
    ref.step(3)
    assert_close(b.field(0, "u"), ref.get(_abi.FIELD_U), PARITY_TOL, "u at t_end")


@pytest.mark.gpu
def test_batch_graph_replay_equals_direct_launches(oracle):
    cfgs = mixed_batch(oracle)[:3]
    a = BatchedIncompressibleSolver(cfgs, autotune=False, use_graph=True)
    b = BatchedIncompressibleSolver(cfgs, autotune=False, use_graph=False)
    assert a.tuning()["graph_nodes"] >= 9 and b.tuning()["graph_nodes"] == 0
    a.advance(3)
    b.advance(3)
    for i in range(len(cfgs)):
        for _, name in FIELDS:
            np.testing.assert_array_equal(a.field(i, name), b.field(i, name))


@pytest.mark.gpu
def test_batch_autotune_keeps_results(oracle):
    cfgs = mixed_batch(oracle)[:3]
    a = BatchedIncompressibleSolver(cfgs, autotune=True)
    t = a.tuning()
    assert all(x in (256, 512, 1024, 2048, 4096) for x in t["tile_elems"])
    assert t["pressure_blocks"] >= len(cfgs) and t["tune_ms"] > 0.0
    a.advance(3)
    refs = oracle_runs(oracle, cfgs, 3)
    for i, (ref, _) in enumerate(refs):
        for fid, name in FIELDS:
            assert_close(a.field(i, name), ref.get(fid), PARITY_TOL, f"instance {i} {name}")


# ---- config checks: these run before any device call ----

def _expect(status, cfgs):
    with pytest.raises(SolverError) as e:
        BatchedIncompressibleSolver(cfgs, autotune=False)
    assert e.value.status == status, str(e.value)
    return str(e.value)


def test_batch_rejects_3d_and_simple_and_mixed_precisions(oracle):
    c2 = cfg2d(oracle, 16, 16)
    c3 = oracle.default_config(3)
    msg = _expect(_abi.ERR_UNSUPPORTED, [c2, c3])
    assert "instance 1" in msg and "2D" in msg
    simple = cfg2d(oracle, 16, 16, coupling=_abi.COUPLING_SIMPLE)
    assert "projection" in _expect(_abi.ERR_UNSUPPORTED, [simple])
    m = cfg2d(oracle, 16, 16, precision=_abi.PRECISION_MIXED)
    assert "precision" in _expect(_abi.ERR_UNSUPPORTED, [c2, m])
    bad = cfg2d(oracle, 2, 16)
    assert "at least 4" in _expect(_abi.ERR_INVALID_CONFIG, [c2, bad])
