"""Host-side mirror of the reference structured solvers, driving the CUDA backend.

Names, fields and error behaviour follow the reference:
  * ``LidDrivenCavity3DConfig`` / ``LidDrivenCavity3DSolver``
    (src/solver/incompressible_3d.rs:8-162),
  * ``SimulationConfig`` / ``IncompressibleSolver`` / ``SolverStep``
    (src/solver/incompressible.rs:58-90, 211-229, 294-586).
``new`` validates like the reference and raises ``SolverError`` with the
reference's message where the reference returns ``Err(String)``. Every call
goes through the C ABI of libflursys_cuda.so (include/flursys_cuda.h).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _abi

_D = C.POINTER(C.c_double)
from .cases import Case, CavityCase, SolverBoundaryOverrides


class SolverError(RuntimeError):
    """The reference's ``Err(String)``; ``status`` is the FlursysStatus code."""

    def __init__(self, message: str, status: int = _abi.ERR_INVALID_CONFIG):
        super().__init__(message)
        self.status = status


def _check(lib, handle, status: int) -> None:
    if status == _abi.OK:
        return
    buf = C.create_string_buffer(1024)
    if handle:
        lib.flursys_cuda_last_error(handle, buf, len(buf))
    else:
        lib.flursys_cuda_global_error(buf, len(buf))
    raise SolverError(buf.value.decode(errors="replace") or _abi.STATUS_NAMES.get(status, str(status)), status)


@dataclass
class BackendOptions:
    """Backend knobs with no reference counterpart."""
    precision: str = "f64"              # "f64" (parity) or "mixed"
    stop_rule: Optional[str] = None     # "abs-inf" | "rel-l2" | "reference-residual"; None = solver default
    pressure_atol: float = 0.0          # rel-l2 absolute part
    pressure_rtol: float = 1.0e-8       # rel-l2 relative part
    residual_replacement_every: int = 50
    device: int = 0
    fcg_weights_path: Optional[str] = None

    def apply(self, cfg: _abi.CudaConfig) -> None:
        cfg.precision = {"f64": _abi.PRECISION_F64, "mixed": _abi.PRECISION_MIXED}[self.precision]
        if self.stop_rule is not None:
            cfg.stop_rule = {"abs-inf": _abi.STOP_ABS_INF, "rel-l2": _abi.STOP_REL_L2,
                             "reference-residual": _abi.STOP_REFERENCE_RESIDUAL}[self.stop_rule]
        cfg.pressure_atol = self.pressure_atol
        cfg.pressure_rtol = self.pressure_rtol
        cfg.residual_replacement_every = self.residual_replacement_every
        cfg.device = self.device
        if self.fcg_weights_path:
            cfg.fcg_weights_path = os.fsencode(self.fcg_weights_path)


# --------------------------------------------------------------------------
# 3D: LidDrivenCavity3DConfig / LidDrivenCavity3DSolver
# --------------------------------------------------------------------------
@dataclass
class LidDrivenCavity3DConfig:
    """src/solver/incompressible_3d.rs:8-47 (same fields and defaults)."""
    nx: int = 32
    ny: int = 32
    nz: int = 32
    length: float = 1.0
    height: float = 1.0
    depth: float = 1.0
    density: float = 1.0
    lid_velocity: float = 1.0
    reynolds: float = 100.0
    dt: float = 5.0e-4
    max_steps: int = 10_000
    pressure_max_iters: int = 2_000
    pressure_tolerance: float = 1.0e-6
    pressure_omega: float = 1.7
    output_dir: str = "results/cavity-3d"
    # backend selection: "sor" mirrors the reference; "pcg" / "fcg" are the
    # Krylov solves of the pinned system.
    pressure_solver: str = "sor"
    backend: BackendOptions = field(default_factory=BackendOptions)

    def viscosity(self) -> float:
        return self.lid_velocity * self.length / self.reynolds

    def to_c(self) -> _abi.CudaConfig:
        lib = _abi.load()
        cfg = _abi.CudaConfig()
        _check(lib, None, lib.flursys_cuda_default_config(3, C.byref(cfg)))
        cfg.nx, cfg.ny, cfg.nz = self.nx, self.ny, self.nz
        cp = cfg.case_params
        cp.length, cp.height, cp.depth = self.length, self.height, self.depth
        cp.density = self.density
        cp.reference_velocity = self.lid_velocity
        cp.reynolds = self.reynolds
        cp.kinematic_viscosity = self.viscosity()
        cfg.dt = self.dt
        cfg.max_steps = self.max_steps
        cfg.pressure_max_iters = self.pressure_max_iters
        cfg.pressure_tolerance = self.pressure_tolerance
        cfg.pressure_omega = self.pressure_omega
        cfg.pressure_solver = {"pcg": _abi.PRESSURE_PCG, "sor": _abi.PRESSURE_SOR,
                               "fcg": _abi.PRESSURE_FCG}[self.pressure_solver]
        cfg.stop_rule = _abi.STOP_REFERENCE_RESIDUAL if self.pressure_solver == "sor" else _abi.STOP_REL_L2
        self.backend.apply(cfg)
        return cfg


@dataclass
class RunSummary3D:
    """src/solver/incompressible_3d.rs:91-99."""
    steps: int
    final_time: float
    max_divergence: float
    pressure_residual: float
    max_speed: float
    elapsed: float


class _Handle:
    """Owns one FlursysCudaHandle."""

    def __init__(self, cfg: _abi.CudaConfig):
        self.lib = _abi.load()
        self._weights = cfg.fcg_weights_path  # keep the bytes alive during create
        h = C.c_void_p()
        _check(self.lib, None, self.lib.flursys_cuda_create(C.byref(cfg), C.byref(h)))
        self.h = h

    def close(self) -> None:
        if self.h:
            self.lib.flursys_cuda_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int = 1) -> _abi.StepReport:
        rep = _abi.StepReport()
        _check(self.lib, self.h, self.lib.flursys_cuda_step(self.h, n, C.byref(rep)))
        return rep

    def field_size(self, fid: int) -> int:
        return int(self.lib.flursys_cuda_field_size(self.h, fid))

    def download(self, fid: int, out: Optional[np.ndarray] = None) -> np.ndarray:
        n = self.field_size(fid)
        if out is None:
            out = np.empty(n, dtype=np.float64)
        _check(self.lib, self.h, self.lib.flursys_cuda_download(self.h, fid, _abi.dptr(out), n))
        return out

    def upload(self, fid: int, values: np.ndarray) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64).ravel()
        _check(self.lib, self.h, self.lib.flursys_cuda_upload(self.h, fid, _abi.dptr(a), a.size))

    def solve_kind(self) -> int:
        """FlursysSolveKind of a 3D handle's pressure solve."""
        k = C.c_int32()
        _check(self.lib, self.h, self.lib.flursys_cuda_solve_kind(self.h, C.byref(k)))
        return int(k.value)

    def snapshot_begin(self, fids) -> "Snapshot":
        """Starts an asynchronous copy of the fields `fids` into page-locked
        host arrays; the next steps run while it drains (Snapshot.wait())."""
        return Snapshot(self, list(fids))

    def set_stream(self, stream_ptr: int) -> None:
        _check(self.lib, self.h, self.lib.flursys_cuda_set_stream(self.h, C.c_void_p(stream_ptr)))

    def state(self):
        s = C.c_int64()
        t = C.c_double()
        self.lib.flursys_cuda_state(self.h, C.byref(s), C.byref(t))
        return s.value, t.value


class Snapshot:
    """A field snapshot draining on the handle's copy stream
    (flursys_cuda_snapshot_begin / _wait). wait() returns {field id: array}."""

    def __init__(self, handle: "_Handle", fids):
        import torch  # page-locked host memory
        self._h = handle
        self.fids = fids
        self._host = [torch.empty(handle.field_size(f), dtype=torch.float64).pin_memory() for f in fids]
        ids = (C.c_int32 * len(fids))(*fids)
        ptrs = (_D * len(fids))(*[C.cast(t.data_ptr(), _D) for t in self._host])
        sizes = (C.c_size_t * len(fids))(*[t.numel() for t in self._host])
        _check(handle.lib, handle.h, handle.lib.flursys_cuda_snapshot_begin(handle.h, ids, len(fids), ptrs, sizes))
        self._done = False

    def wait(self) -> dict:
        if not self._done:
            _check(self._h.lib, self._h.h, self._h.lib.flursys_cuda_snapshot_wait(self._h.h))
            self._done = True
        return {f: t.numpy() for f, t in zip(self.fids, self._host)}


class LidDrivenCavity3DSolver:
    """src/solver/incompressible_3d.rs:117-172 on the device."""

    def __init__(self, cfg: LidDrivenCavity3DConfig):
        self.cfg = cfg
        self._h = _Handle(cfg.to_c())
        self.last_report: Optional[_abi.StepReport] = None

    @classmethod
    def new(cls, cfg: LidDrivenCavity3DConfig) -> "LidDrivenCavity3DSolver":
        return cls(cfg)

    @property
    def handle(self) -> _Handle:
        return self._h

    def advance(self, steps: int = 1) -> _abi.StepReport:
        self.last_report = self._h.step(steps)
        return self.last_report

    def run(self, write_output: bool = True) -> RunSummary3D:
        """run() (:136-162): max_steps steps, then field.vtk in output_dir."""
        started = time.perf_counter()
        rep = self.advance(self.cfg.max_steps)
        if write_output:
            from . import output
            os.makedirs(self.cfg.output_dir, exist_ok=True)
            output.write_legacy_vtk_3d(os.path.join(self.cfg.output_dir, "field.vtk"),
                                       "FLURSYS 3D lid-driven cavity", self)
        return RunSummary3D(steps=int(rep.iteration), final_time=rep.time,
                            max_divergence=rep.continuity_residual,
                            pressure_residual=rep.pressure_residual, max_speed=rep.max_speed,
                            elapsed=time.perf_counter() - started)

    def field(self, name: str) -> np.ndarray:
        fid = {"u": _abi.FIELD_U, "v": _abi.FIELD_V, "w": _abi.FIELD_W, "pressure": _abi.FIELD_PRESSURE,
               "rhs": _abi.FIELD_RHS, "u_star": _abi.FIELD_U_STAR, "v_star": _abi.FIELD_V_STAR,
               "w_star": _abi.FIELD_W_STAR}[name]
        return self._h.download(fid)

    def close(self) -> None:
        self._h.close()


# --------------------------------------------------------------------------
# 2D: SimulationConfig / IncompressibleSolver
# --------------------------------------------------------------------------
@dataclass
class TimeStepSettings:
    """src/solver/incompressible.rs:35-56."""
    adaptive: bool = False
    min_dt: float = 1.0e-6
    max_dt: float = 1.0e-2
    target_cfl: float = 0.5
    target_diffusion_number: float = 0.25
    max_growth_factor: float = 1.1


@dataclass
class ThermalBoundaryCondition:
    """src/physics.rs:17-25: "adiabatic" or "fixed-temperature" with its value."""
    kind: str = "adiabatic"
    temperature: float = 0.0

    @classmethod
    def fixed(cls, temperature: float) -> "ThermalBoundaryCondition":
        return cls("fixed-temperature", temperature)


@dataclass
class ThermalSettings:
    """src/physics.rs:27-56 (same fields and defaults)."""
    model: str = "off"  # "off" | "constant-properties"
    initial_temperature: float = 293.15
    thermal_diffusivity: float = 2.2e-5
    source_temperature_rate: float = 0.0
    left: ThermalBoundaryCondition = field(default_factory=ThermalBoundaryCondition)
    right: ThermalBoundaryCondition = field(default_factory=ThermalBoundaryCondition)
    bottom: ThermalBoundaryCondition = field(default_factory=ThermalBoundaryCondition)
    top: ThermalBoundaryCondition = field(default_factory=ThermalBoundaryCondition)


@dataclass
class BoussinesqBuoyancy:
    """BuoyancyModel::Boussinesq (src/physics.rs:59-70): g * beta * (T - T_ref)."""
    reference_temperature: float = 293.15
    thermal_expansion: float = 3.4e-3
    gravity_x: float = 0.0
    gravity_y: float = -9.81


@dataclass
class PhysicsSettings:
    """src/physics.rs:72-77; `buoyancy` is None for BuoyancyModel::Off."""
    thermal: ThermalSettings = field(default_factory=ThermalSettings)
    buoyancy: Optional[BoussinesqBuoyancy] = None

    def fill(self, ph: _abi.PhysicsSettings) -> None:
        t = self.thermal
        ph.energy_model = {"off": _abi.ENERGY_OFF, "constant-properties": _abi.ENERGY_CONSTANT_PROPERTIES}[t.model]
        ph.initial_temperature = t.initial_temperature
        ph.thermal_diffusivity = t.thermal_diffusivity
        ph.source_temperature_rate = t.source_temperature_rate
        for side, bc in enumerate([t.left, t.right, t.bottom, t.top]):
            ph.thermal[side].kind = {"adiabatic": _abi.THERMAL_ADIABATIC,
                                     "fixed-temperature": _abi.THERMAL_FIXED_TEMPERATURE}[bc.kind]
            ph.thermal[side].temperature = bc.temperature
        if self.buoyancy is None:
            ph.buoyancy = _abi.BUOYANCY_OFF
        else:
            b = self.buoyancy
            ph.buoyancy = _abi.BUOYANCY_BOUSSINESQ
            ph.reference_temperature = b.reference_temperature
            ph.thermal_expansion = b.thermal_expansion
            ph.gravity_x, ph.gravity_y = b.gravity_x, b.gravity_y


@dataclass
class SimulationConfig:
    """src/solver/incompressible.rs:58-90."""
    case: Case = field(default_factory=lambda: Case.lid_driven_cavity(CavityCase()))
    nx: int = 64
    ny: int = 64
    dt: float = 1.0e-3
    time_step: TimeStepSettings = field(default_factory=TimeStepSettings)
    max_steps: int = 100_000
    t_end: float = 100.0
    convection: str = "upwind"          # "upwind" | "central"
    coupling: str = "projection"        # "projection" | "simple"
    pressure_solver: str = "pcg"        # "pcg" | "sor"
    pressure_max_iters: int = 1200
    pressure_tolerance: float = 1.0e-5
    pressure_omega: float = 1.7
    velocity_relaxation: float = 0.7
    pressure_relaxation: float = 0.3
    print_every: int = 100
    output_every: int = 100
    frame_every: int = 500
    steady_tolerance: float = 1.0e-7
    minimum_steps: int = 2000
    threads: int = 0
    boundary_overrides: SolverBoundaryOverrides = field(default_factory=SolverBoundaryOverrides)
    physics: PhysicsSettings = field(default_factory=PhysicsSettings)
    output_dir: str = "results/cavity"
    backend: BackendOptions = field(default_factory=BackendOptions)

    def to_c(self) -> _abi.CudaConfig:
        lib = _abi.load()
        cfg = _abi.CudaConfig()
        _check(lib, None, lib.flursys_cuda_default_config(2, C.byref(cfg)))
        self.case.fill(cfg.case_params)
        self.boundary_overrides.fill(cfg.overrides)
        cfg.nx, cfg.ny, cfg.nz = self.nx, self.ny, 1
        cfg.dt = self.dt
        ts = self.time_step
        cfg.adaptive = 1 if ts.adaptive else 0
        cfg.min_dt, cfg.max_dt = ts.min_dt, ts.max_dt
        cfg.target_cfl, cfg.target_diffusion_number = ts.target_cfl, ts.target_diffusion_number
        cfg.max_growth_factor = ts.max_growth_factor
        cfg.max_steps = self.max_steps
        cfg.t_end = self.t_end
        cfg.convection = {"upwind": _abi.CONVECTION_UPWIND, "first-order-upwind": _abi.CONVECTION_UPWIND,
                          "central": _abi.CONVECTION_CENTRAL}[self.convection]
        cfg.coupling = {"projection": _abi.COUPLING_PROJECTION, "simple": _abi.COUPLING_SIMPLE}[self.coupling]
        cfg.pressure_solver = {"pcg": _abi.PRESSURE_PCG, "sor": _abi.PRESSURE_SOR,
                               "fcg": _abi.PRESSURE_FCG}[self.pressure_solver]
        cfg.stop_rule = _abi.STOP_ABS_INF
        cfg.pressure_max_iters = self.pressure_max_iters
        cfg.pressure_tolerance = self.pressure_tolerance
        cfg.pressure_omega = self.pressure_omega
        cfg.velocity_relaxation = self.velocity_relaxation
        cfg.pressure_relaxation = self.pressure_relaxation
        cfg.steady_tolerance = self.steady_tolerance
        cfg.minimum_steps = self.minimum_steps
        self.physics.fill(cfg.physics)
        self.backend.apply(cfg)
        return cfg


@dataclass
class SolverStep:
    """src/solver/incompressible.rs:211-229."""
    iteration: int
    time: float
    time_step: float
    continuity_residual: float
    pressure_residual: float
    pressure_iterations: int
    momentum_residual: float
    max_speed: float
    momentum_cfl: float
    viscous_diffusion_number: float
    drag_coefficient: float
    lift_coefficient: float
    converged: bool
    reached_end_time: bool

    @classmethod
    def from_report(cls, r: _abi.StepReport) -> "SolverStep":
        return cls(int(r.iteration), r.time, r.time_step, r.continuity_residual, r.pressure_residual,
                   int(r.pressure_iterations), r.momentum_residual, r.max_speed, r.momentum_cfl,
                   r.viscous_diffusion_number, r.drag_coefficient, r.lift_coefficient, bool(r.converged),
                   bool(r.reached_end_time))


@dataclass
class RunSummary:
    """src/solver/incompressible.rs:200-209."""
    case_name: str
    steps: int
    final_time: float
    max_divergence: float
    pressure_residual: float
    elapsed: float
    converged: bool


@dataclass
class FieldUpdate:
    """src/solver/incompressible.rs:231-244."""
    nx: int
    ny: int
    pressure: np.ndarray
    speed: np.ndarray
    velocity_x: np.ndarray
    velocity_y: np.ndarray
    vorticity: np.ndarray
    solid: np.ndarray
    temperature: Optional[np.ndarray] = None


class IncompressibleSolver:
    """src/solver/incompressible.rs:319-586 on the device."""

    def __init__(self, cfg: SimulationConfig):
        self.cfg = cfg
        self._h = _Handle(cfg.to_c())
        self.last_report: Optional[_abi.StepReport] = None

    @classmethod
    def new(cls, cfg: SimulationConfig) -> "IncompressibleSolver":
        return cls(cfg)

    @property
    def handle(self) -> _Handle:
        return self._h

    def advance(self) -> SolverStep:
        """advance() (:523-555): one step and its SolverStep."""
        self.last_report = self._h.step(1)
        return SolverStep.from_report(self.last_report)

    def run(self, write_output: bool = False) -> RunSummary:
        """run() (:368-499): steps until max_steps, t_end or steady. With
        `write_output`, every `output_every` steps (and at the end) a field
        snapshot is taken on the device and drained to the host while the
        next steps run; a writer thread turns it into frames/field_NNNNN.vtk
        and field.csv / field.vtk of the last one (output.rs:31-125)."""
        from concurrent.futures import ThreadPoolExecutor
        started = time.perf_counter()
        step, _ = self._h.state()
        rep = None
        converged = False
        every = max(1, int(self.cfg.output_every)) if write_output else 1 << 20
        pool = ThreadPoolExecutor(max_workers=1) if write_output else None
        pending = []
        if write_output:
            os.makedirs(os.path.join(self.cfg.output_dir, "frames"), exist_ok=True)

        def emit(pfu, frame):
            fu = pfu.wait()
            from . import output
            output.write_legacy_vtk(os.path.join(self.cfg.output_dir, "frames", f"field_{frame:05d}.vtk"),
                                    self.cfg.case.name(), self, fu)
            return fu

        frame = 0
        while step < self.cfg.max_steps:
            chunk = min(self.cfg.max_steps - step, every - step % every)
            rep = self._h.step(chunk)
            step = int(rep.iteration)
            done = bool(rep.converged) or bool(rep.reached_end_time) or step >= self.cfg.max_steps
            if write_output and (step % every == 0 or done):
                pending.append(pool.submit(emit, self.field_update_async(), frame))
                frame += 1
            if rep.converged:
                converged = True
                break
            if rep.reached_end_time:
                break
        if write_output:
            last = None
            for f in pending:
                last = f.result()
            pool.shutdown()
            if last is not None:
                from . import output
                output.write_field_csv(os.path.join(self.cfg.output_dir, "field.csv"), self, last)
                output.write_legacy_vtk(os.path.join(self.cfg.output_dir, "field.vtk"), self.cfg.case.name(), self,
                                        last)
        self.last_report = rep
        return RunSummary(case_name=self.cfg.case.name(), steps=step, final_time=rep.time if rep else 0.0,
                          max_divergence=rep.continuity_residual if rep else 0.0,
                          pressure_residual=rep.pressure_residual if rep else 0.0,
                          elapsed=time.perf_counter() - started, converged=converged)

    def field(self, name: str) -> np.ndarray:
        fid = {"u": _abi.FIELD_U, "v": _abi.FIELD_V, "pressure": _abi.FIELD_PRESSURE, "rhs": _abi.FIELD_RHS,
               "u_star": _abi.FIELD_U_STAR, "v_star": _abi.FIELD_V_STAR, "speed": _abi.FIELD_SPEED,
               "vorticity": _abi.FIELD_VORTICITY, "u_cell": _abi.FIELD_U_CELL,
               "v_cell": _abi.FIELD_V_CELL, "temperature": _abi.FIELD_TEMPERATURE}[name]
        return self._h.download(fid)

    def field_update_async(self) -> "PendingFieldUpdate":
        """field_update() taken without stalling the solver: the fields are
        copied on the device after the work already enqueued and drained to
        page-locked host memory on a copy stream; .wait() gives the
        FieldUpdate."""
        fids = [_abi.FIELD_U, _abi.FIELD_V, _abi.FIELD_PRESSURE, _abi.FIELD_SPEED, _abi.FIELD_VORTICITY]
        if self.cfg.physics.thermal.model == "constant-properties":
            fids.append(_abi.FIELD_TEMPERATURE)
        return PendingFieldUpdate(self, self._h.snapshot_begin(fids))

    def field_update(self) -> FieldUpdate:
        """field_update() (:563-586)."""
        nx, ny = self.cfg.nx, self.cfg.ny
        u = self.field("u").reshape(ny, nx + 1)
        v = self.field("v").reshape(ny + 1, nx)
        return FieldUpdate(nx=nx, ny=ny, pressure=self.field("pressure"), speed=self.field("speed"),
                           velocity_x=(0.5 * (u[:, :-1] + u[:, 1:])).ravel(),
                           velocity_y=(0.5 * (v[:-1, :] + v[1:, :])).ravel(),
                           vorticity=self.field("vorticity"),
                           solid=self.cfg.case.solid_mask(nx, ny).ravel(),
                           temperature=self.field("temperature")
                           if self.cfg.physics.thermal.model == "constant-properties" else None)

    def close(self) -> None:
        self._h.close()


class PendingFieldUpdate:
    """A FieldUpdate whose fields are still draining to the host."""

    def __init__(self, solver: "IncompressibleSolver", snap: Snapshot):
        self._solver = solver
        self._snap = snap

    def wait(self) -> FieldUpdate:
        f = self._snap.wait()
        cfg = self._solver.cfg
        nx, ny = cfg.nx, cfg.ny
        u = f[_abi.FIELD_U].reshape(ny, nx + 1)
        v = f[_abi.FIELD_V].reshape(ny + 1, nx)
        return FieldUpdate(nx=nx, ny=ny, pressure=f[_abi.FIELD_PRESSURE].copy(), speed=f[_abi.FIELD_SPEED].copy(),
                           velocity_x=(0.5 * (u[:, :-1] + u[:, 1:])).ravel(),
                           velocity_y=(0.5 * (v[:-1, :] + v[1:, :])).ravel(),
                           vorticity=f[_abi.FIELD_VORTICITY].copy(), solid=cfg.case.solid_mask(nx, ny).ravel(),
                           temperature=f[_abi.FIELD_TEMPERATURE].copy() if _abi.FIELD_TEMPERATURE in f else None)


class BatchedIncompressibleSolver:
    """Many independent IncompressibleSolver instances (2D, projection
    coupling) of uneven size advanced together on one device.

    No reference counterpart: each instance computes what
    ``IncompressibleSolver`` (src/solver/incompressible.rs:294-746) computes
    for its config. ``advance(n)`` steps every instance that is still active;
    an instance whose time reached t_end, or whose step failed, stops and
    reports its status through ``status(i)``.
    """

    def __init__(self, configs, autotune: bool = True, use_graph: bool = True):
        if not configs:
            raise SolverError("a batch needs at least one config", _abi.ERR_INVALID_ARGUMENT)
        self.lib = _abi.load()
        self.configs = list(configs)
        arr = (_abi.CudaConfig * len(self.configs))()
        for i, c in enumerate(self.configs):
            arr[i] = c.to_c() if hasattr(c, "to_c") else c
        flags = (_abi.BATCH_AUTOTUNE if autotune else 0) | (0 if use_graph else _abi.BATCH_NO_GRAPH)
        h = C.c_void_p()
        _check(self.lib, None, self.lib.flursys_cuda_batch_create(arr, len(self.configs), flags, C.byref(h)))
        self.h = h

    def __len__(self) -> int:
        return len(self.configs)

    def advance(self, nsteps: int = 1) -> None:
        _check(self.lib, None, self.lib.flursys_cuda_batch_step(self.h, int(nsteps)))

    def report(self, i: int) -> _abi.StepReport:
        rep = _abi.StepReport()
        st = C.c_int32()
        _check(self.lib, None, self.lib.flursys_cuda_batch_report(self.h, i, C.byref(rep), C.byref(st)))
        return rep

    def status(self, i: int) -> int:
        rep = _abi.StepReport()
        st = C.c_int32()
        _check(self.lib, None, self.lib.flursys_cuda_batch_report(self.h, i, C.byref(rep), C.byref(st)))
        return int(st.value)

    def step_report(self, i: int) -> SolverStep:
        return SolverStep.from_report(self.report(i))

    def field(self, i: int, name: str) -> np.ndarray:
        cfg = self.configs[i]
        nx, ny = cfg.nx, cfg.ny
        fid = {"u": _abi.FIELD_U, "v": _abi.FIELD_V, "pressure": _abi.FIELD_PRESSURE, "rhs": _abi.FIELD_RHS,
               "u_star": _abi.FIELD_U_STAR, "v_star": _abi.FIELD_V_STAR, "speed": _abi.FIELD_SPEED,
               "vorticity": _abi.FIELD_VORTICITY, "u_cell": _abi.FIELD_U_CELL,
               "v_cell": _abi.FIELD_V_CELL}[name]
        n = {"u": (nx + 1) * ny, "v": nx * (ny + 1), "u_star": (nx + 1) * ny, "v_star": nx * (ny + 1)}.get(name, nx * ny)
        out = np.empty(n, dtype=np.float64)
        _check(self.lib, None, self.lib.flursys_cuda_batch_download(self.h, i, fid, _abi.dptr(out), n))
        return out

    def tuning(self) -> dict:
        t = _abi.BatchTuning()
        _check(self.lib, None, self.lib.flursys_cuda_batch_tuning(self.h, C.byref(t)))
        return {"tile_elems": list(t.tile_elems), "pressure_blocks_per_sm": t.pressure_blocks_per_sm,
                "pressure_blocks": t.pressure_blocks, "graph_nodes": t.graph_nodes, "tune_ms": t.tune_ms}

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.flursys_cuda_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class ChannelSimpleConfig:
    """The steady plane-channel case of solve_incompressible
    (src/unstructured_incompressible.rs:368-482) on nx x ny uniform quads,
    with IncompressibleSolverOptions defaults (:38-49). Re is on the mean
    velocity (2/3 of the parabolic peak) and the height, as
    src/project.rs:497-509 defines it."""
    nx: int = 2048
    ny: int = 512
    length: float = 8.0
    height: float = 1.0
    reynolds: float = 200.0
    inlet_peak_velocity: float = 1.0
    outlet_pressure: float = 0.0
    max_outer_iterations: int = 200
    continuity_tolerance: float = 1.0e-10
    velocity_relaxation: float = 0.7
    pressure_relaxation: float = 0.3
    momentum_solver: tuple = (1.0e-10, 1.0e-8, 1000)   # (atol, rtol, max_iterations)
    pressure_solver: tuple = (1.0e-10, 1.0e-8, 1000)

    def kinematic_viscosity(self) -> float:
        return (2.0 / 3.0) * self.inlet_peak_velocity * self.height / self.reynolds

    def to_c(self) -> _abi.SimpleConfig:
        lib = _abi.load()
        c = _abi.SimpleConfig()
        _check(lib, None, lib.flursys_cuda_simple_default_config(C.byref(c)))
        c.nx, c.ny = self.nx, self.ny
        c.length, c.height = self.length, self.height
        c.kinematic_viscosity = self.kinematic_viscosity()
        c.inlet_peak_velocity = self.inlet_peak_velocity
        c.outlet_pressure = self.outlet_pressure
        c.max_outer_iterations = self.max_outer_iterations
        c.continuity_tolerance = self.continuity_tolerance
        c.velocity_relaxation = self.velocity_relaxation
        c.pressure_relaxation = self.pressure_relaxation
        c.momentum_solver = _abi.LinearSolverOptions(*self.momentum_solver)
        c.pressure_solver = _abi.LinearSolverOptions(*self.pressure_solver)
        return c


def solve_simple_channel(cfg) -> dict:
    """flursys_cuda_simple_channel: cell velocity, pressure, face fluxes
    (+x x-faces then +y y-faces), continuity history and the report."""
    lib = _abi.load()
    c = cfg.to_c() if hasattr(cfg, "to_c") else cfg
    n = c.nx * c.ny
    u, v, p = np.zeros(n), np.zeros(n), np.zeros(n)
    flux = np.zeros((c.nx + 1) * c.ny + c.nx * (c.ny + 1))
    hist = np.zeros(c.max_outer_iterations + 1)
    rep = _abi.SimpleReport()
    _check(lib, None, lib.flursys_cuda_simple_channel(C.byref(c), _abi.dptr(u), _abi.dptr(v), _abi.dptr(p),
                                                      _abi.dptr(flux), _abi.dptr(hist), C.byref(rep)))
    return {"u": u, "v": v, "p": p, "flux": flux, "history": hist[:rep.outer_iterations + 1], "report": rep}
