"""2D structured solver: CUDA backend (through the C ABI) against the FP64
oracle of src/solver/incompressible.rs, on every case and option of the path."""
import ctypes as C

import numpy as np
import pytest

from flursys_b200 import _abi
from flursys_b200.solver import SolverError, _Handle

from .paritylib import assert_close, rel_l2
from .test_oracle_solver import case_cfg

pytestmark = pytest.mark.gpu

PARITY_TOL = 1e-10
FIELDS = [(_abi.FIELD_U, "u"), (_abi.FIELD_V, "v"), (_abi.FIELD_PRESSURE, "p"), (_abi.FIELD_SPEED, "speed"),
          (_abi.FIELD_VORTICITY, "vorticity")]


def cfg2d(oracle, nx, ny, tol=1e-13, steps=5, dt=1e-3, **kw):
    cfg = oracle.default_config(2)
    cfg.nx, cfg.ny = nx, ny
    cfg.dt = dt
    cfg.t_end = 100.0
    cfg.max_steps = steps
    cfg.pressure_tolerance = tol
    cfg.pressure_max_iters = 20000
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


def run_pair(oracle, cfg, steps):
    ref = oracle.OracleSolver(cfg)
    gpu = _Handle(cfg)
    for _ in range(steps):
        a = ref.step(1)
        b = gpu.step(1)
        assert a.iteration == b.iteration
        assert abs(a.time - b.time) <= 1e-15 * max(1.0, abs(a.time))
        assert abs(a.time_step - b.time_step) <= 1e-15
    return ref, gpu, a, b


def check_fields(ref, gpu, tol=PARITY_TOL, fields=FIELDS):
    for fid, name in fields:
        assert_close(gpu.download(fid), ref.get(fid), tol, name)


@pytest.mark.parametrize("shape,convection", [((16, 16), _abi.CONVECTION_UPWIND), ((48, 40), _abi.CONVECTION_UPWIND),
                                              ((32, 32), _abi.CONVECTION_CENTRAL)])
def test_cavity_steps_match_oracle(oracle, shape, convection):
    cfg = cfg2d(oracle, *shape, convection=convection)
    ref, gpu, a, b = run_pair(oracle, cfg, 5)
    check_fields(ref, gpu)
    # max|div| after projection is rounding noise (~1e-14); compare it on the scale of 1/dx
    assert abs(a.continuity_residual - b.continuity_residual) <= 1e-11 * shape[0]
    assert abs(a.max_speed - b.max_speed) <= 1e-12
    assert abs(a.momentum_residual - b.momentum_residual) <= 1e-10 * max(1e-12, a.momentum_residual)
    assert abs(a.momentum_cfl - b.momentum_cfl) <= 1e-12


# The 70x8 backward step (35 x 2 domain) is badly conditioned: with the
# solve stopped at max|r| < 1e-12 the pressure itself is only determined to
# about 1e-12 / lambda_min ~ 1e-9 relative, whichever reduction order is used.
@pytest.mark.parametrize("kind,nx,ny,ptol", [(_abi.CASE_CYLINDER, 80, 32, 1e-10),
                                             (_abi.CASE_BACKWARD_STEP, 70, 8, 1e-8),
                                             (_abi.CASE_CHANNEL, 80, 16, 1e-10)])
def test_solid_and_outlet_cases_match_oracle(oracle, kind, nx, ny, ptol):
    # tests/smoke.rs:57-111 shapes; tight PCG so the fields compare at 1e-10
    cfg = case_cfg(oracle, kind, nx, ny)
    cfg.pressure_tolerance = 1e-12
    cfg.pressure_max_iters = 20000
    cfg.t_end = 100.0
    ref, gpu, a, b = run_pair(oracle, cfg, 3)
    check_fields(ref, gpu, fields=[f for f in FIELDS if f[1] != "p"])
    assert_close(gpu.download(_abi.FIELD_PRESSURE), ref.get(_abi.FIELD_PRESSURE), ptol, "p")
    assert b.continuity_residual < 1e-5
    if kind == _abi.CASE_CYLINDER:
        assert abs(a.drag_coefficient - b.drag_coefficient) <= 1e-9 * max(1.0, abs(a.drag_coefficient))
        assert abs(a.lift_coefficient - b.lift_coefficient) <= 1e-9 * max(1.0, abs(a.lift_coefficient))


def test_simple_coupling_matches_oracle(oracle):
    cfg = cfg2d(oracle, 16, 16, coupling=_abi.COUPLING_SIMPLE, t_end=0.0, minimum_steps=1)
    ref, gpu, a, b = run_pair(oracle, cfg, 3)
    check_fields(ref, gpu)
    assert not b.reached_end_time and b.iteration == 3


def test_adaptive_time_step_matches_oracle(oracle):
    cfg = cfg2d(oracle, 32, 32, adaptive=1, dt=1e-3, min_dt=1e-6, max_dt=1e-2)
    ref, gpu, a, b = run_pair(oracle, cfg, 6)
    check_fields(ref, gpu)
    assert abs(a.time_step - b.time_step) <= 1e-15


def test_rel_l2_stop_rule_and_mixed_precision(oracle):
    # config-1 shape of the solve (Jacobi-PCG to 1e-8 relative) on a 64^2 cavity
    cfg = cfg2d(oracle, 64, 64, stop_rule=_abi.STOP_REL_L2, pressure_rtol=1e-8)
    cfgm = cfg2d(oracle, 64, 64, stop_rule=_abi.STOP_REL_L2, pressure_rtol=1e-8, precision=_abi.PRECISION_MIXED)
    ref = oracle.OracleSolver(cfg)
    g64 = _Handle(cfg)
    gmx = _Handle(cfgm)
    for _ in range(5):
        a, b, m = ref.step(1), g64.step(1), gmx.step(1)
        assert abs(a.pressure_iterations - b.pressure_iterations) <= 1
        assert m.pressure_true_relative_residual <= 1e-8 * 1.0001
    assert_close(g64.download(_abi.FIELD_U), ref.get(_abi.FIELD_U), 1e-7, "u f64")
    for fid in (_abi.FIELD_U, _abi.FIELD_V):
        assert rel_l2(gmx.download(fid), ref.get(fid)) <= 1e-6


def test_red_black_sor_converges_to_the_same_system(oracle):
    cfg = cfg2d(oracle, 24, 24, pressure_solver=_abi.PRESSURE_SOR, tol=1e-11)
    ref = oracle.OracleSolver(cfg)
    gpu = _Handle(cfg)
    a, b = ref.step(2), gpu.step(2)
    assert b.pressure_residual < 1e-11
    assert rel_l2(gpu.download(_abi.FIELD_U), ref.get(_abi.FIELD_U)) < 1e-8


def test_end_time_semantics(oracle):
    # incompressible.rs:2617-2636
    cfg = cfg2d(oracle, 8, 8, dt=1e-3, t_end=2.5e-3, tol=1e-4)
    cfg.pressure_max_iters = 50
    gpu = _Handle(cfg)
    rep = gpu.step(1)
    while not rep.reached_end_time:
        rep = gpu.step(1)
    assert abs(rep.time - 2.5e-3) < 1e-12
    with pytest.raises(SolverError) as e:
        gpu.step(1)
    assert str(e.value) == "projection simulation has already reached t_end"
    assert e.value.status == _abi.ERR_REACHED_END_TIME


def test_boundary_override_sets_the_face_velocity(oracle):
    # incompressible.rs:2703-2720
    cfg = cfg2d(oracle, 64, 64)
    cfg.overrides[_abi.SIDE_LEFT].kind = _abi.BOUNDARY_VELOCITY
    cfg.overrides[_abi.SIDE_LEFT].u = 1.75
    gpu = _Handle(cfg)
    assert gpu.download(_abi.FIELD_U).reshape(64, 65)[32, 0] == 1.75
    ref = oracle.OracleSolver(cfg)
    ref.step(2)
    gpu.step(2)
    check_fields(ref, gpu)


@pytest.mark.parametrize("precision", [_abi.PRECISION_F64, _abi.PRECISION_MIXED])
def test_stencil_pcg_2d_entry_matches_oracle(oracle, cudalib, precision):
    nx, ny = 40, 24
    rng = np.random.default_rng(5)
    rhs = rng.standard_normal(nx * ny)
    rhs -= rhs.mean()
    opts = _abi.LinearSolverOptions(0.0, 1e-10, 5000)
    st, xref, rref = oracle.stencil_pcg(nx, ny, 1, 1 / nx, 1 / ny, 1.0, rhs, np.zeros_like(rhs), opts)
    assert st == 0
    x = np.zeros_like(rhs)
    rep = _abi.LinearSolveReport()
    st = cudalib.flursys_cuda_stencil_pcg(nx, ny, 1, 1 / nx, 1 / ny, 1.0, _abi.dptr(rhs), _abi.dptr(x), precision,
                                          C.byref(opts), C.byref(rep))
    assert st == 0 and rep.status == _abi.LINEAR_CONVERGED
    assert rel_l2(x, xref) < (1e-9 if precision == _abi.PRECISION_F64 else 1e-7)


@pytest.mark.parametrize("precision", [_abi.PRECISION_F64, _abi.PRECISION_MIXED])
def test_cluster_and_grid_barrier_paths_agree(oracle, monkeypatch, precision):
    # A 128^2 cavity without solids runs its pressure solve as one thread-block
    # cluster (hardware cluster barrier); FLURSYS_2D_CLUSTER=0 forces the
    # software grid barrier. Same system, same stop rule: same iteration
    # counts and fields to rounding.
    cfg = cfg2d(oracle, 128, 128, stop_rule=_abi.STOP_REL_L2, pressure_rtol=1e-8, precision=precision)
    runs = []
    for env in ("1", "0"):
        monkeypatch.setenv("FLURSYS_2D_CLUSTER", env)
        g = _Handle(cfg)
        reps = [g.step(1) for _ in range(3)]
        runs.append((reps, {fid: g.download(fid) for fid, _ in FIELDS[:3]}))
    monkeypatch.delenv("FLURSYS_2D_CLUSTER")
    (rc, fc), (rg, fg) = runs
    for a, b in zip(rc, rg):
        assert a.pressure_status == b.pressure_status == _abi.LINEAR_CONVERGED
        assert abs(a.pressure_iterations - b.pressure_iterations) <= 1
    for fid, name in FIELDS[:3]:
        assert rel_l2(fc[fid], fg[fid]) <= (1e-10 if precision == _abi.PRECISION_F64 else 1e-6), name
