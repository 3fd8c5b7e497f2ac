"""Pins the oracle's restatement of the structured solvers to the reference's
own known-answer and smoke tests (src/solver/incompressible.rs:2417-2720,
tests/smoke.rs:9-155)."""
import ctypes as C

import numpy as np
import pytest

from flursys_b200 import _abi


def stability(oracle, *args):
    cfl, dnu = C.c_double(), C.c_double()
    oracle.load().orc_momentum_stability_numbers(*args, C.byref(cfl), C.byref(dnu))
    return cfl.value, dnu.value


def adaptive(oracle, current, mu, mv, dx, dy, nu, thermal, min_dt, max_dt, cfl, diff, growth):
    out = C.c_double()
    msg = C.create_string_buffer(512)
    st = oracle.load().orc_adaptive_time_step(current, mu, mv, dx, dy, nu, thermal, min_dt, max_dt, cfl, diff,
                                              growth, C.byref(out), msg, 512)
    return st, out.value, msg.value.decode()


def test_momentum_stability_numbers_match_known_values(oracle):
    cfl, dnu = stability(oracle, 0.01, 0.1, 0.5, 0.25, 2.0, 1.0)
    assert abs(cfl - 0.08) < 1e-12 and abs(dnu - 0.02) < 1e-12
    cfl, dnu = stability(oracle, 0.1, 0.25, 0.5, 0.25, 0.0, 0.0)
    assert cfl == 0.0 and abs(dnu - 0.5) < 1e-12
    a, _ = stability(oracle, 0.1, 0.2, 0.5, 0.25, 2.0, 1.0)
    b, _ = stability(oracle, 0.1, 0.2, 0.25, 0.5, 1.0, 2.0)
    assert abs(a - b) < 1e-12


def test_adaptive_time_step_known_answers(oracle):
    # incompressible.rs:2444-2583
    st, dt, _ = adaptive(oracle, 0.1, 2.0, 1.0, 0.5, 0.25, 1e-3, -1, 1e-3, 1.0, 0.5, 0.5, 10.0)
    assert st == 0 and abs(dt - 0.0625) < 1e-12
    st, dt, _ = adaptive(oracle, 0.5, 0.0, 0.0, 0.5, 0.25, 0.1, -1, 1e-3, 1.0, 1.0, 0.25, 10.0)
    assert st == 0 and abs(dt - 0.125) < 1e-12
    st, dt, _ = adaptive(oracle, 0.5, 0.0, 0.0, 0.5, 0.25, 0.1, 0.4, 1e-3, 1.0, 1.0, 0.25, 10.0)
    assert st == 0 and abs(dt - 0.03125) < 1e-12
    st, dt, _ = adaptive(oracle, 0.1, 0.0, 0.0, 1.0, 1.0, 1e-3, -1, 1e-3, 0.8, 1.0, 0.25, 1.1)
    assert st == 0 and abs(dt - 0.11) < 1e-12
    st, _, msg = adaptive(oracle, 0.5, 0.0, 0.0, 0.5, 0.25, 0.1, -1, 0.2, 1.0, 1.0, 0.25, 10.0)
    assert st != 0 and "required stable time step" in msg and "min_dt" in msg


def cavity_cfg(oracle, nx, ny, dt=1e-3, t_end=1e-3, its=800, tol=1e-6):
    cfg = oracle.default_config(2)
    cfg.nx, cfg.ny, cfg.dt, cfg.t_end = nx, ny, dt, t_end
    cfg.max_steps = 1
    cfg.pressure_max_iters = its
    cfg.pressure_tolerance = tol
    cfg.steady_tolerance = 1e-10
    cfg.minimum_steps = 100
    return cfg


def test_projection_step_reports_when_the_physical_end_time_is_reached(oracle):
    # incompressible.rs:2617-2636 (8x8, dt 1e-3, t_end 2.5e-3, PCG 50 its, tol 1e-4)
    cfg = cavity_cfg(oracle, 8, 8, t_end=2.5e-3, its=50, tol=1e-4)
    s = oracle.OracleSolver(cfg)
    rep = s.step(1)
    while not rep.reached_end_time:
        rep = s.step(1)
    assert abs(rep.time - 2.5e-3) < 1e-12
    with pytest.raises(oracle.OracleError) as e:
        s.step(1)
    assert str(e.value) == "projection simulation has already reached t_end"


def test_simple_steps_do_not_report_end_time(oracle):
    cfg = cavity_cfg(oracle, 8, 8, its=50, tol=1e-4)
    cfg.coupling = _abi.COUPLING_SIMPLE
    cfg.t_end = 0.0
    rep = oracle.OracleSolver(cfg).step(1)
    assert not rep.reached_end_time and rep.iteration == 1


def test_default_time_step_settings_preserve_fixed_step_behavior(oracle):
    cfg = cavity_cfg(oracle, 8, 8, t_end=0.002, its=20, tol=1e-4)
    s = oracle.OracleSolver(cfg)
    a = s.step(1)
    b = s.step(1)
    assert abs(a.time - 1e-3) < 1e-12 and abs(b.time - 2e-3) < 1e-12
    assert abs(a.time_step - 1e-3) < 1e-12 and abs(b.time_step - 1e-3) < 1e-12


def test_project_boundary_override_sets_the_solver_face_velocity(oracle):
    # incompressible.rs:2703-2720: Velocity{u: 1.75} on the left face
    cfg = cavity_cfg(oracle, 64, 64)
    cfg.overrides[_abi.SIDE_LEFT].kind = _abi.BOUNDARY_VELOCITY
    cfg.overrides[_abi.SIDE_LEFT].u = 1.75
    s = oracle.OracleSolver(cfg)
    u = s.get(_abi.FIELD_U).reshape(64, 65)
    assert u[32, 0] == 1.75


def case_cfg(oracle, kind, nx, ny):
    cfg = cavity_cfg(oracle, nx, ny)
    cp = cfg.case_params
    cp.kind = kind
    if kind == _abi.CASE_CYLINDER:
        cp.length, cp.height, cp.density, cp.reference_velocity = 25.0, 10.0, 1.0, 1.0
        cp.cylinder_xc, cp.cylinder_yc, cp.cylinder_diameter = 5.0, 5.0, 1.0
        cp.cylinder_perturbation, cp.cylinder_mu, cp.kinematic_viscosity = 1e-3, 0.01, 0.01
    elif kind == _abi.CASE_BACKWARD_STEP:
        cp.length, cp.height, cp.step_height, cp.step_x = 35.0, 2.0, 1.0, 5.0
        cp.reference_velocity, cp.kinematic_viscosity = 1.0, 0.01
    elif kind == _abi.CASE_CHANNEL:
        cp.length, cp.height, cp.reference_velocity, cp.kinematic_viscosity = 10.0, 1.0, 1.0, 0.01
    return cfg


@pytest.mark.parametrize("kind,nx,ny", [(_abi.CASE_CAVITY, 16, 16), (_abi.CASE_CYLINDER, 80, 32),
                                        (_abi.CASE_BACKWARD_STEP, 70, 8), (_abi.CASE_CHANNEL, 80, 16)])
def test_cases_advance_one_step(oracle, kind, nx, ny):
    # tests/smoke.rs:57-111
    rep = oracle.OracleSolver(case_cfg(oracle, kind, nx, ny)).step(1)
    assert np.isfinite(rep.continuity_residual) and rep.continuity_residual < 1e-5


def test_simple_coupling_advances_a_steady_iteration(oracle):
    # tests/smoke.rs:38-55
    cfg = cavity_cfg(oracle, 16, 16)
    cfg.coupling = _abi.COUPLING_SIMPLE
    cfg.max_steps, cfg.t_end, cfg.minimum_steps = 2, 0.0, 1
    s = oracle.OracleSolver(cfg)
    rep = s.step(2)
    assert rep.iteration == 2 and rep.continuity_residual < 1e-5 and rep.pressure_residual < 1e-5


def test_cavity_3d_advances_divergence_free_flow(oracle):
    # tests/smoke.rs:113-130 (8^3, 2 steps, dt 5e-4, default SOR)
    cfg = oracle.default_config(3)
    cfg.nx = cfg.ny = cfg.nz = 8
    cfg.max_steps = 2
    s = oracle.OracleSolver(cfg)
    rep = s.step(2)
    assert rep.iteration == 2
    assert np.isfinite(rep.continuity_residual) and rep.continuity_residual < 1e-5
    assert rep.max_speed > 0.0


def test_multithreaded_pcg_matches_single_thread(oracle):
    # tests/smoke.rs:132-155 (32x32, 3 steps, 1 vs 4 threads)
    cfg = cavity_cfg(oracle, 32, 32, t_end=3e-3)
    try:
        oracle.set_threads(1)
        a = oracle.OracleSolver(cfg).step(3)
        oracle.set_threads(4)
        b = oracle.OracleSolver(cfg).step(3)
    finally:
        oracle.set_threads(1)
    assert a.iteration == b.iteration == 3
    assert abs(a.continuity_residual - b.continuity_residual) < 1e-10
    assert abs(a.pressure_residual - b.pressure_residual) < 1e-10


def test_3d_pcg_and_sor_solve_the_same_pinned_system(oracle):
    """The 3D PCG oracle converges to the system the reference's SOR solves."""
    cfg = oracle.default_config(3)
    cfg.nx = cfg.ny = cfg.nz = 8
    cfg.pressure_tolerance = 1e-11
    cfg.pressure_max_iters = 20000
    s_sor = oracle.OracleSolver(cfg)
    s_sor.step(1)
    cfg2 = oracle.default_config(3)
    cfg2.nx = cfg2.ny = cfg2.nz = 8
    cfg2.pressure_solver = _abi.PRESSURE_PCG
    cfg2.stop_rule = _abi.STOP_REL_L2
    cfg2.pressure_rtol = 1e-14
    s_pcg = oracle.OracleSolver(cfg2)
    s_pcg.step(1)
    assert s_pcg.pressure_residual() < 1e-8
    p1, p2 = s_sor.get(_abi.FIELD_PRESSURE), s_pcg.get(_abi.FIELD_PRESSURE)
    assert p1[0] == 0.0 and p2[0] == 0.0
    assert np.max(np.abs(p1 - p2)) <= 1e-9 * max(1.0, np.max(np.abs(p1)))
