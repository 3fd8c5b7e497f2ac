"""Canonical cases and boundary overrides (src/cases/*.rs, src/preprocess.rs:1331-1406).

Each case keeps the reference's fields and defaults and fills the POD
``FlursysCaseParams`` of the C ABI. Kinematic viscosity is derived the way
the reference derives it (CavityCase::default, project.rs:480-509).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _abi


@dataclass
class CavityCase:
    """src/cases/cavity.rs:1-26."""
    length: float = 1.0
    height: float = 1.0
    rho: float = 1.0
    lid_velocity: float = 1.0
    reynolds: float = 100.0
    nu: Optional[float] = None

    def __post_init__(self):
        if self.nu is None:
            self.nu = self.lid_velocity * self.length / self.reynolds


@dataclass
class ChannelCase:
    """src/cases/channel.rs:1-25."""
    length: float = 10.0
    height: float = 1.0
    rho: float = 1.0
    u_mean: float = 1.0
    reynolds: float = 100.0
    nu: Optional[float] = None

    def __post_init__(self):
        if self.nu is None:
            self.nu = self.u_mean * self.height / self.reynolds


@dataclass
class CylinderCase:
    """src/cases/cylinder.rs:1-34."""
    length: float = 25.0
    height: float = 10.0
    diameter: float = 1.0
    xc: float = 5.0
    yc: float = 5.0
    rho: float = 1.0
    u_inf: float = 1.0
    reynolds: float = 100.0
    mu: float = 0.01
    nu: float = 0.01
    perturbation: float = 1.0e-3


@dataclass
class BackwardStepCase:
    """src/cases/backward_step.rs:1-30."""
    length: float = 35.0
    height: float = 2.0
    step_height: float = 1.0
    step_x: float = 5.0
    rho: float = 1.0
    u_mean: float = 1.0
    reynolds: float = 100.0
    nu: Optional[float] = None

    def __post_init__(self):
        if self.nu is None:
            self.nu = self.u_mean * self.step_height / self.reynolds


class Case:
    """src/cases/mod.rs:45-244: the case enum."""

    def __init__(self, kind: int, data):
        self.kind = kind
        self.data = data

    @classmethod
    def lid_driven_cavity(cls, c: CavityCase) -> "Case":
        return cls(_abi.CASE_CAVITY, c)

    @classmethod
    def cylinder(cls, c: CylinderCase) -> "Case":
        return cls(_abi.CASE_CYLINDER, c)

    @classmethod
    def backward_facing_step(cls, c: BackwardStepCase) -> "Case":
        return cls(_abi.CASE_BACKWARD_STEP, c)

    @classmethod
    def channel(cls, c: ChannelCase) -> "Case":
        return cls(_abi.CASE_CHANNEL, c)

    def name(self) -> str:
        return {_abi.CASE_CAVITY: "Lid-Driven Cavity", _abi.CASE_CYLINDER: "Cylinder Flow Re=100",
                _abi.CASE_BACKWARD_STEP: "Backward-Facing Step Flow",
                _abi.CASE_CHANNEL: "Plane Poiseuille Channel Flow"}[self.kind]

    def domain(self):
        return self.data.length, self.data.height

    def density(self) -> float:
        return self.data.rho

    def kinematic_viscosity(self) -> float:
        return self.data.nu

    def is_solid(self, x: float, y: float) -> bool:
        """Case::is_solid (mod.rs:218-227)."""
        d = self.data
        if self.kind == _abi.CASE_CYLINDER:
            return (x - d.xc) ** 2 + (y - d.yc) ** 2 <= (0.5 * d.diameter) ** 2
        if self.kind == _abi.CASE_BACKWARD_STEP:
            return x < d.step_x and y < d.step_height
        return False

    def solid_mask(self, nx: int, ny: int) -> np.ndarray:
        length, height = self.domain()
        dx, dy = length / nx, height / ny
        m = np.zeros((ny, nx), dtype=bool)
        for j in range(ny):
            for i in range(nx):
                m[j, i] = self.is_solid((i + 0.5) * dx, (j + 0.5) * dy)
        return m

    def fill(self, cp: _abi.CaseParams) -> None:
        d = self.data
        cp.kind = self.kind
        cp.length, cp.height = d.length, d.height
        cp.depth = 1.0
        cp.density = d.rho
        cp.kinematic_viscosity = d.nu
        cp.reynolds = d.reynolds
        if self.kind == _abi.CASE_CAVITY:
            cp.reference_velocity = d.lid_velocity
        elif self.kind == _abi.CASE_CYLINDER:
            cp.reference_velocity = d.u_inf
            cp.cylinder_xc, cp.cylinder_yc = d.xc, d.yc
            cp.cylinder_diameter, cp.cylinder_perturbation, cp.cylinder_mu = d.diameter, d.perturbation, d.mu
        elif self.kind == _abi.CASE_BACKWARD_STEP:
            cp.reference_velocity = d.u_mean
            cp.step_x, cp.step_height = d.step_x, d.step_height
        else:
            cp.reference_velocity = d.u_mean


@dataclass
class SolverBoundaryOverride:
    """SolverBoundaryOverride (preprocess.rs:1356-1361)."""
    kind: int = _abi.BOUNDARY_VELOCITY
    u: float = 0.0
    v: float = 0.0
    pressure: float = 0.0

    @classmethod
    def velocity(cls, u: float, v: float) -> "SolverBoundaryOverride":
        return cls(_abi.BOUNDARY_VELOCITY, u, v, 0.0)

    @classmethod
    def pressure_outlet(cls, pressure: float) -> "SolverBoundaryOverride":
        return cls(_abi.BOUNDARY_PRESSURE_OUTLET, 0.0, 0.0, pressure)

    @classmethod
    def symmetry(cls) -> "SolverBoundaryOverride":
        return cls(_abi.BOUNDARY_SYMMETRY)


@dataclass
class SolverBoundaryOverrides:
    """SolverBoundaryOverrides (preprocess.rs:1363-1406); None keeps the case default."""
    left: Optional[SolverBoundaryOverride] = None
    right: Optional[SolverBoundaryOverride] = None
    bottom: Optional[SolverBoundaryOverride] = None
    top: Optional[SolverBoundaryOverride] = None

    def fill(self, arr) -> None:
        for side, ov in enumerate((self.left, self.right, self.bottom, self.top)):
            o = arr[side]
            if ov is None:
                o.kind, o.u, o.v, o.pressure = _abi.BOUNDARY_CASE_DEFAULT, 0.0, 0.0, 0.0
            else:
                o.kind, o.u, o.v, o.pressure = ov.kind, ov.u, ov.v, ov.pressure
