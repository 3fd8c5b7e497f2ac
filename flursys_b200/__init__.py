"""B200 (sm_100a) backend for the FLURSYS structured MAC projection step.

The compute path is libflursys_cuda.so (hand-written CUDA behind the C ABI of
include/flursys_cuda.h). This package is its host-side mirror of the
reference's solver and linear-algebra interfaces; it has no CPU fallback.
"""
from . import _abi
from .cases import (BackwardStepCase, Case, CavityCase, ChannelCase, CylinderCase, SolverBoundaryOverride,
                    SolverBoundaryOverrides)
from .solver import (BackendOptions, BatchedIncompressibleSolver, BoussinesqBuoyancy, FieldUpdate, IncompressibleSolver,
                     LidDrivenCavity3DConfig, LidDrivenCavity3DSolver, PhysicsSettings, RunSummary, RunSummary3D,
                     SimulationConfig, SolverError, SolverStep, ThermalBoundaryCondition, ThermalSettings,
                     TimeStepSettings)

__all__ = [
    "BackendOptions", "BatchedIncompressibleSolver", "BackwardStepCase", "Case", "CavityCase", "ChannelCase", "CylinderCase", "FieldUpdate",
    "IncompressibleSolver", "LidDrivenCavity3DConfig", "LidDrivenCavity3DSolver", "RunSummary", "RunSummary3D",
    "SimulationConfig", "SolverBoundaryOverride", "SolverBoundaryOverrides", "SolverError", "SolverStep",
    "TimeStepSettings", "load_library", "BoussinesqBuoyancy", "PhysicsSettings", "ThermalBoundaryCondition",
    "ThermalSettings",
]


def load_library():
    """Loads libflursys_cuda.so; raises ImportError when it was not built."""
    return _abi.load()
