"""Energy equation and Boussinesq buoyancy: pins the oracle's restatement to
the reference's own thermal tests (src/solver/incompressible.rs:2501-2529,
2722-2802; src/project.rs:819-832) and checks that the CUDA library's config
validation gives the reference's messages (no device needed)."""
import ctypes as C

import numpy as np
import pytest

from flursys_b200 import _abi


def thermal_test_cfg(oracle):
    """fixed_temperature_boundary_diffuses_into_the_domain (:2723-2750)."""
    cfg = oracle.default_config(2)
    cfg.nx = cfg.ny = 16
    cfg.dt = 1.0e-4
    cfg.max_steps = 2
    cfg.t_end = 2.0e-4
    cfg.convection = _abi.CONVECTION_UPWIND
    cfg.pressure_solver = _abi.PRESSURE_PCG
    cfg.pressure_max_iters = 50
    cfg.pressure_tolerance = 1.0e-4
    cfg.pressure_omega = 1.5
    ph = cfg.physics
    ph.energy_model = _abi.ENERGY_CONSTANT_PROPERTIES
    ph.initial_temperature = 300.0
    ph.thermal_diffusivity = 1.0e-3
    ph.thermal[_abi.SIDE_BOTTOM].kind = _abi.THERMAL_FIXED_TEMPERATURE
    ph.thermal[_abi.SIDE_BOTTOM].temperature = 400.0
    return cfg


def example_cfg(oracle):
    """examples/thermal-buoyancy-cavity.flursys.json: 48^2 cavity, lid 0.1,
    Re 100, dt 1e-4, left 303.15 K, right 283.15 K, Boussinesq, g = -9.81."""
    cfg = oracle.default_config(2)
    cfg.nx = cfg.ny = 48
    cp = cfg.case_params
    cp.reference_velocity = 0.1
    cp.reynolds = 100.0
    cp.kinematic_viscosity = 0.1 * 1.0 / 100.0
    cfg.dt = 1.0e-4
    cfg.pressure_tolerance = 1.0e-6
    cfg.pressure_max_iters = 1200
    ph = cfg.physics
    ph.energy_model = _abi.ENERGY_CONSTANT_PROPERTIES
    ph.initial_temperature = 293.15
    ph.thermal_diffusivity = 2.0e-5
    ph.thermal[_abi.SIDE_LEFT].kind = _abi.THERMAL_FIXED_TEMPERATURE
    ph.thermal[_abi.SIDE_LEFT].temperature = 303.15
    ph.thermal[_abi.SIDE_RIGHT].kind = _abi.THERMAL_FIXED_TEMPERATURE
    ph.thermal[_abi.SIDE_RIGHT].temperature = 283.15
    ph.buoyancy = _abi.BUOYANCY_BOUSSINESQ
    ph.reference_temperature = 293.15
    ph.thermal_expansion = 0.0034
    ph.gravity_x, ph.gravity_y = 0.0, -9.81
    return cfg


def create_error(oracle, cfg):
    try:
        oracle.OracleSolver(cfg)
    except oracle.OracleError as e:
        return e.status, str(e)
    return 0, ""


def product_create_error(cfg):
    lib = _abi.load()
    h = C.c_void_p()
    st = lib.flursys_cuda_create(C.byref(cfg), C.byref(h))
    buf = C.create_string_buffer(512)
    lib.flursys_cuda_global_error(buf, 512)
    return st, buf.value.decode()


def test_fixed_temperature_boundary_diffuses_into_the_domain(oracle):
    ref = oracle.OracleSolver(thermal_test_cfg(oracle))
    ref.step(1)
    t = ref.get(_abi.FIELD_TEMPERATURE).reshape(16, 16)  # [j, i]
    assert t[0, 8] > 300.0
    assert abs(t[8, 8] - 300.0) < 1.0e-9


def test_buoyancy_cannot_be_enabled_without_energy_transport(oracle):
    cfg = oracle.default_config(2)
    cfg.nx = cfg.ny = 16
    cfg.physics.buoyancy = _abi.BUOYANCY_BOUSSINESQ
    cfg.physics.reference_temperature = 293.15
    cfg.physics.thermal_expansion = 3.4e-3
    cfg.physics.gravity_y = -9.81
    st, msg = create_error(oracle, cfg)
    assert st == _abi.ERR_INVALID_CONFIG and "requires the constant-property energy equation" in msg
    assert product_create_error(cfg) == (st, msg)


def test_adaptive_time_step_uses_thermal_diffusivity_when_larger(oracle):
    out = C.c_double()
    msg = C.create_string_buffer(256)
    st = oracle.load().orc_adaptive_time_step(0.5, 0.0, 0.0, 0.5, 0.25, 0.1, 0.4, 1e-3, 1.0, 1.0, 0.25, 10.0,
                                              C.byref(out), msg, 256)
    assert st == 0 and abs(out.value - 0.03125) < 1e-12


def test_thermal_buoyancy_example_validates_and_runs(oracle):
    cfg = example_cfg(oracle)
    ref = oracle.OracleSolver(cfg)
    ref.step(5)
    t = ref.get(_abi.FIELD_TEMPERATURE).reshape(48, 48)
    # heated left wall, cooled right wall
    assert t[:, 0].mean() > 293.15 > t[:, -1].mean()
    # the body force is g * beta * (T - T_ref) as the reference writes it
    # (:843-845, :908-910): with g_y < 0 it pushes the fluid at the heated
    # wall along -y relative to the same run without buoyancy
    quiet = example_cfg(oracle)
    quiet.physics.buoyancy = _abi.BUOYANCY_OFF
    ref0 = oracle.OracleSolver(quiet)
    ref0.step(5)
    v, v0 = ref.get(_abi.FIELD_V).reshape(49, 48), ref0.get(_abi.FIELD_V).reshape(49, 48)
    assert v[24, 0] < v0[24, 0] and v[24, -1] > v0[24, -1]


@pytest.mark.parametrize("case", ["fourier", "nonfinite", "boundary", "boussinesq", "three_d"])
def test_validation_messages_match_between_oracle_and_library(oracle, case):
    cfg = thermal_test_cfg(oracle)
    if case == "fourier":
        cfg.physics.thermal_diffusivity = 1.0
        cfg.dt = 1e-3
        cfg.t_end = 1.0
        expect = "explicit thermal diffusion is unstable: alpha*dt*(1/dx^2 + 1/dy^2)=5.120e-1 exceeds 0.5"
    elif case == "nonfinite":
        cfg.physics.source_temperature_rate = float("inf")
        expect = ("thermal initial temperature, diffusivity, and source must be finite; diffusivity must be "
                  "positive")
    elif case == "boundary":
        cfg.physics.thermal[_abi.SIDE_TOP].kind = _abi.THERMAL_FIXED_TEMPERATURE
        cfg.physics.thermal[_abi.SIDE_TOP].temperature = float("nan")
        expect = "fixed thermal boundary temperatures must be finite"
    elif case == "boussinesq":
        cfg.physics.buoyancy = _abi.BUOYANCY_BOUSSINESQ
        cfg.physics.thermal_expansion = -1.0
        expect = ("Boussinesq reference temperature, expansion coefficient, and gravity must be finite; "
                  "expansion must be non-negative")
    else:
        cfg = oracle.default_config(3)
        cfg.physics.energy_model = _abi.ENERGY_CONSTANT_PROPERTIES
        expect = ("the current 3D backend supports constant-property flow only; thermal and buoyancy models "
                  "are not available")
    st, msg = create_error(oracle, cfg)
    assert msg == expect and st != 0
    assert product_create_error(cfg) == (st, msg)


def test_adaptive_dt_message_uses_rust_exponent_format(oracle):
    out = C.c_double()
    msg = C.create_string_buffer(512)
    st = oracle.load().orc_adaptive_time_step(0.5, 0.0, 0.0, 0.5, 0.25, 0.1, -1, 0.2, 1.0, 1.0, 0.25, 10.0,
                                              C.byref(out), msg, 512)
    assert st != 0
    assert msg.value.decode() == ("required stable time step 1.250e-1 is below configured min_dt 2.000e-1; "
                                  "CFL constraint=1.000e0, diffusion constraint=1.250e-1")
