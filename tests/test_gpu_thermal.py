"""Energy equation and Boussinesq buoyancy on the device (2D handle) against
the FP64 oracle of src/solver/incompressible.rs:748-922 (buoyancy in the
predictor) and :1441-1530 (advance_temperature), through the C ABI."""
import numpy as np
import pytest

from flursys_b200 import _abi
from flursys_b200.solver import SolverError, _Handle

from .paritylib import assert_close
from .test_oracle_solver import case_cfg
from .test_oracle_thermal import example_cfg, thermal_test_cfg

pytestmark = pytest.mark.gpu

PARITY_TOL = 1e-10
FIELDS = [(_abi.FIELD_U, "u"), (_abi.FIELD_V, "v"), (_abi.FIELD_PRESSURE, "p"), (_abi.FIELD_SPEED, "speed"),
          (_abi.FIELD_TEMPERATURE, "temperature")]


def tight(cfg):
    cfg.pressure_tolerance = 1e-13
    cfg.pressure_max_iters = 20000
    return cfg


def run_pair(oracle, cfg, steps):
    ref = oracle.OracleSolver(cfg)
    gpu = _Handle(cfg)
    for _ in range(steps):
        a, b = ref.step(1), gpu.step(1)
        assert a.iteration == b.iteration and abs(a.time_step - b.time_step) <= 1e-15
    for fid, name in FIELDS:
        assert_close(gpu.download(fid), ref.get(fid), PARITY_TOL, name)
    return ref, gpu


def test_thermal_buoyancy_cavity_matches_oracle(oracle):
    run_pair(oracle, tight(example_cfg(oracle)), 20)


def test_fixed_temperature_boundary_matches_oracle_and_reference_gate(oracle):
    ref, gpu = run_pair(oracle, thermal_test_cfg(oracle), 2)
    t = gpu.download(_abi.FIELD_TEMPERATURE).reshape(16, 16)
    assert t[0, 8] > 300.0 and abs(t[8, 8] - 300.0) < 1e-9


def test_source_buoyancy_x_adaptive_and_solid_body_match_oracle(oracle):
    # cylinder case: solid cells keep their temperature and mirror the centre
    # for their fluid neighbours; a heat source; gravity along x; adaptive
    # dt whose diffusion limit is set by alpha > nu
    cfg = tight(case_cfg(oracle, _abi.CASE_CYLINDER, 80, 32))
    cfg.t_end = 100.0
    cfg.adaptive = 1
    cfg.dt = 1e-3
    cfg.min_dt = 1e-6
    ph = cfg.physics
    ph.energy_model = _abi.ENERGY_CONSTANT_PROPERTIES
    ph.initial_temperature = 290.0
    ph.thermal_diffusivity = 3.0 * cfg.case_params.kinematic_viscosity
    ph.source_temperature_rate = 5.0
    ph.thermal[_abi.SIDE_LEFT].kind = _abi.THERMAL_FIXED_TEMPERATURE
    ph.thermal[_abi.SIDE_LEFT].temperature = 310.0
    ph.thermal[_abi.SIDE_TOP].kind = _abi.THERMAL_FIXED_TEMPERATURE
    ph.thermal[_abi.SIDE_TOP].temperature = 280.0
    ph.buoyancy = _abi.BUOYANCY_BOUSSINESQ
    ph.reference_temperature = 295.0
    ph.thermal_expansion = 0.01
    ph.gravity_x, ph.gravity_y = 2.0, -9.81
    run_pair(oracle, cfg, 8)


def test_thermal_cfl_error_matches_oracle(oracle):
    cfg = oracle.default_config(2)
    cfg.nx = cfg.ny = 16
    cfg.dt = 0.2
    cfg.t_end = 100.0
    cfg.pressure_tolerance = 1e-12
    cfg.pressure_max_iters = 5000
    cfg.physics.energy_model = _abi.ENERGY_CONSTANT_PROPERTIES
    cfg.physics.thermal_diffusivity = 1e-3
    ref = oracle.OracleSolver(cfg)
    gpu = _Handle(cfg)
    t_before = gpu.download(_abi.FIELD_TEMPERATURE)
    with pytest.raises(oracle.OracleError) as a:
        ref.step(1)
    with pytest.raises(SolverError) as b:
        gpu.step(1)
    assert str(a.value).startswith("explicit thermal advection is unstable at step 1: CFL=")
    assert str(b.value) == str(a.value)
    # the temperature is not advanced, the velocity is (as in the reference)
    assert np.array_equal(gpu.download(_abi.FIELD_TEMPERATURE), t_before)
    assert_close(gpu.download(_abi.FIELD_U), ref.get(_abi.FIELD_U), PARITY_TOL, "u")


def test_field_update_carries_temperature():
    from flursys_b200 import (IncompressibleSolver, PhysicsSettings, SimulationConfig, ThermalBoundaryCondition,
                              ThermalSettings)
    th = ThermalSettings(model="constant-properties", bottom=ThermalBoundaryCondition.fixed(350.0))
    cfg = SimulationConfig(nx=16, ny=16, dt=1e-4, t_end=1.0, physics=PhysicsSettings(thermal=th))
    s = IncompressibleSolver(cfg)
    s.advance()
    fu = s.field_update()
    assert fu.temperature is not None and fu.temperature.shape == (256,)
    assert fu.temperature.max() > 293.15
    s.close()
