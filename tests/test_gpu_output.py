"""Output overlapped with compute: a field snapshot is copied on the device
after the step that produced it and drained to the host while later steps
run (flursys_cuda_snapshot_begin / _wait); the writers of src/output.rs
then see exactly the fields of that step."""
import numpy as np
import pytest

from flursys_b200 import _abi
from flursys_b200.solver import SolverError, _Handle

pytestmark = pytest.mark.gpu


def _cfg(oracle, thermal=False):
    cfg = oracle.default_config(2)
    cfg.nx, cfg.ny = 48, 40
    cfg.t_end = 100.0
    cfg.pressure_tolerance = 1e-10
    cfg.pressure_max_iters = 5000
    if thermal:
        cfg.physics.energy_model = _abi.ENERGY_CONSTANT_PROPERTIES
        cfg.physics.thermal[_abi.SIDE_BOTTOM].kind = _abi.THERMAL_FIXED_TEMPERATURE
        cfg.physics.thermal[_abi.SIDE_BOTTOM].temperature = 320.0
    return cfg


@pytest.mark.parametrize("thermal", [False, True])
def test_snapshot_holds_the_fields_of_its_step_while_later_steps_run(oracle, thermal):
    fids = [_abi.FIELD_U, _abi.FIELD_V, _abi.FIELD_PRESSURE, _abi.FIELD_SPEED, _abi.FIELD_VORTICITY]
    if thermal:
        fids.append(_abi.FIELD_TEMPERATURE)
    a, b = _Handle(_cfg(oracle, thermal)), _Handle(_cfg(oracle, thermal))
    a.step(3)
    snap = a.snapshot_begin(fids)
    a.step(4)  # runs while the snapshot drains
    got = snap.wait()
    b.step(3)
    for f in fids:
        assert np.array_equal(got[f], b.download(f)), f
    b.step(4)
    assert np.array_equal(a.download(_abi.FIELD_U), b.download(_abi.FIELD_U))


def test_one_pending_snapshot_per_handle(oracle):
    a = _Handle(_cfg(oracle))
    a.step(1)
    s1 = a.snapshot_begin([_abi.FIELD_PRESSURE])
    with pytest.raises(SolverError):
        a.snapshot_begin([_abi.FIELD_U])
    s1.wait()
    a.snapshot_begin([_abi.FIELD_U]).wait()


def test_run_writes_frames_and_final_fields_from_snapshots(tmp_path):
    from flursys_b200 import IncompressibleSolver, PhysicsSettings, SimulationConfig, ThermalSettings
    from flursys_b200 import output
    th = ThermalSettings(model="constant-properties")
    cfg = SimulationConfig(nx=32, ny=32, dt=1e-3, t_end=1.0, max_steps=12, output_every=5,
                           output_dir=str(tmp_path / "cavity"), physics=PhysicsSettings(thermal=th))
    s = IncompressibleSolver(cfg)
    summary = s.run(write_output=True)
    assert summary.steps == 12
    frames = sorted((tmp_path / "cavity" / "frames").iterdir())
    assert [f.name for f in frames] == ["field_00000.vtk", "field_00001.vtk", "field_00002.vtk"]
    ref = tmp_path / "ref.csv"
    output.write_field_csv(str(ref), s)  # synchronous download of the final state
    assert (tmp_path / "cavity" / "field.csv").read_text() == ref.read_text()
    assert (tmp_path / "cavity" / "field.csv").read_text().splitlines()[0].endswith(",temperature")
    assert "SCALARS temperature double 1" in (tmp_path / "cavity" / "field.vtk").read_text()
    s.close()
