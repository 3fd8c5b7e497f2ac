"""3D pressure PCG, MIXED precision, with the solver state resident on the
chip (one cooperative launch per solve; the default where the grid's
32 x 32 x tz tiles fit one per SM): against the FP64 oracle, against the
graph-driven two-launch PCG (FLURSYS_PCG_RESIDENT=0), single-reduction form
(the default for the L2 stop rule) against the two-reduction form
(FLURSYS_PCG_RESIDENT=2, and every other stop rule), at its iteration cap,
and with an injected grid-barrier fault.

Iteration counts of two MIXED solves that differ only in rounding (another
summation order of a dot product, alpha rounded to FP32 for the vector
updates) are compared within a few percent: near its attainable accuracy
the FP32 recurrence amplifies such differences, and convergence is accepted
only at an FP64 residual replacement."""
import numpy as np
import pytest

from flursys_b200 import _abi
from flursys_b200.solver import SolverError, _Handle

from .test_gpu_cavity3d import FIELDS, MIXED_TOL, cfg3d
from .test_gpu_pcg3d_variants import _vel_rel

pytestmark = pytest.mark.gpu


def _close_iterations(a, b):
    return abs(a - b) <= 3 + max(a, b) // 25


def _run(oracle, shape, steps, monkeypatch, resident=True, rtol=1e-8, max_iters=20000, rule=_abi.STOP_REL_L2):
    if resident is False:
        monkeypatch.setenv("FLURSYS_PCG_RESIDENT", "0")
    elif resident == "two":
        monkeypatch.setenv("FLURSYS_PCG_RESIDENT", "2")
    cfg = cfg3d(oracle, *shape, rtol=rtol, precision=_abi.PRECISION_MIXED, rule=rule)
    cfg.pressure_max_iters = max_iters
    if rule != _abi.STOP_REL_L2:
        cfg.pressure_tolerance = rtol
    gpu = _Handle(cfg)
    reps = [gpu.step(1) for _ in range(steps)]
    fields = {fid: gpu.download(fid) for fid, _ in FIELDS}
    monkeypatch.delenv("FLURSYS_PCG_RESIDENT", raising=False)
    return reps, fields, gpu


@pytest.mark.parametrize("shape", [(32, 32, 32), (48, 40, 36), (20, 70, 9), (64, 96, 50)])
def test_resident_pcg_against_fp64_oracle(oracle, monkeypatch, shape):
    ref = oracle.OracleSolver(cfg3d(oracle, *shape, rtol=1e-8))
    steps = 4
    ref_reps = [ref.step(1) for _ in range(steps)]
    reps, fields, _ = _run(oracle, shape, steps, monkeypatch)
    for a, b in zip(reps, ref_reps):
        assert a.pressure_status == _abi.LINEAR_CONVERGED
        assert a.pressure_true_relative_residual <= 1.0e-8 * 1.0001
        # MIXED accepts convergence only at an FP64 residual replacement
        # (every 50 iterations) and its FP32 vectors drift from the FP64
        # recurrence, so it may take up to one replacement interval plus a
        # quarter more iterations than the FP64 oracle, never fewer.
        assert b.pressure_iterations - 3 <= a.pressure_iterations
        assert a.pressure_iterations <= b.pressure_iterations + 50 + b.pressure_iterations // 4
    assert _vel_rel(fields, {fid: ref.get(fid) for fid, _ in FIELDS[:3]}) <= MIXED_TOL


def test_resident_and_graph_paths_agree(oracle, monkeypatch):
    shape = (48, 40, 32)  # > 100 iterations: residual replacements inside each solve
    res, f1, _ = _run(oracle, shape, 3, monkeypatch)
    seq, f2, _ = _run(oracle, shape, 3, monkeypatch, resident=False)
    for a, b in zip(res, seq):
        assert a.pressure_status == b.pressure_status == _abi.LINEAR_CONVERGED
        assert b.pressure_iterations > 100
        assert _close_iterations(a.pressure_iterations, b.pressure_iterations)
    assert _vel_rel(f1, f2) <= MIXED_TOL


@pytest.mark.parametrize("shape", [(48, 40, 32), (64, 96, 50)])
def test_single_and_two_reduction_forms_agree(oracle, monkeypatch, shape):
    one, f1, g1 = _run(oracle, shape, 3, monkeypatch)
    two, f2, g2 = _run(oracle, shape, 3, monkeypatch, resident="two")
    assert g1.solve_kind() == g2.solve_kind() == _abi.SOLVE_RESIDENT
    for a, b in zip(one, two):
        assert a.pressure_status == b.pressure_status == _abi.LINEAR_CONVERGED
        assert a.pressure_true_relative_residual <= 1.0e-8 * 1.0001
        assert _close_iterations(a.pressure_iterations, b.pressure_iterations)
    assert _vel_rel(f1, f2) <= MIXED_TOL


def test_max_norm_stop_rule_runs_resident_two_reduction_form(oracle, monkeypatch):
    shape = (40, 36, 28)
    cfg = cfg3d(oracle, *shape, rule=_abi.STOP_ABS_INF)
    cfg.pressure_tolerance = 1e-7
    ref = oracle.OracleSolver(cfg)
    ref_reps = [ref.step(1) for _ in range(3)]
    reps, fields, gpu = _run(oracle, shape, 3, monkeypatch, rtol=1e-7, rule=_abi.STOP_ABS_INF)
    assert gpu.solve_kind() == _abi.SOLVE_RESIDENT
    for a, b in zip(reps, ref_reps):
        assert a.pressure_status == _abi.LINEAR_CONVERGED
        assert b.pressure_iterations - 3 <= a.pressure_iterations <= b.pressure_iterations + 50 + b.pressure_iterations // 4
    assert _vel_rel(fields, {fid: ref.get(fid) for fid, _ in FIELDS[:3]}) <= MIXED_TOL


def test_resident_iteration_cap(oracle, monkeypatch):
    reps, fields, _ = _run(oracle, (32, 32, 32), 1, monkeypatch, rtol=1e-12, max_iters=37)
    rep = reps[0]
    assert rep.pressure_status == _abi.LINEAR_MAX_ITERATIONS
    assert rep.pressure_iterations == 37
    assert all(np.isfinite(v).all() for v in fields.values())


def test_resident_barrier_timeout_is_reported(oracle, monkeypatch, cudalib):
    reps, _, gpu = _run(oracle, (32, 32, 32), 1, monkeypatch)
    assert cudalib.flursys_cuda_debug_inject_barrier_fault(1) == 0
    with pytest.raises(SolverError) as e:
        gpu.step(1)
    assert e.value.status == _abi.ERR_TIMEOUT and "timed out" in str(e.value)
    rep = gpu.step(1)  # the injection covered one launch; the context is intact
    assert rep.pressure_status == _abi.LINEAR_CONVERGED


@pytest.mark.parametrize("shape", [(64, 40, 48), (132, 20, 12)])  # partial x tiles; short chunks
def test_staged_operand_pass_matches_register_pass(oracle, monkeypatch, shape):
    # graph path (not resident): the cp.async-staged operand kernel (default
    # for MIXED) against the register-prefetch kernel (FLURSYS_STENCIL=vec)
    monkeypatch.setenv("FLURSYS_STENCIL", "vec")
    vec, f2, _ = _run(oracle, shape, 3, monkeypatch, resident=False)
    monkeypatch.delenv("FLURSYS_STENCIL")
    pipe, f1, _ = _run(oracle, shape, 3, monkeypatch, resident=False)
    for a, b in zip(pipe, vec):
        assert a.pressure_status == b.pressure_status == _abi.LINEAR_CONVERGED
        assert _close_iterations(a.pressure_iterations, b.pressure_iterations)
    assert _vel_rel(f1, f2) <= MIXED_TOL
    ref = oracle.OracleSolver(cfg3d(oracle, *shape, rtol=1e-8))
    for _ in range(3):
        ref.step(1)
    assert _vel_rel(f1, {fid: ref.get(fid) for fid, _ in FIELDS[:3]}) <= MIXED_TOL
