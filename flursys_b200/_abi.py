"""ctypes mirror of include/flursys_cuda.h and the loader of libflursys_cuda.so.

The structures below follow the C header field by field; a CPU test compiles
the header and compares every size and offset with these definitions.
Loading fails loudly when the shared library is missing: there is no CPU
fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

ABI_VERSION = 2

# FlursysStatus
OK = 0
ERR_DIMENSION_MISMATCH = 1
ERR_INVALID_CSR = 2
ERR_INDEX_OUT_OF_BOUNDS = 3
ERR_NON_FINITE = 4
ERR_MISSING_DIAGONAL = 5
ERR_ZERO_DIAGONAL = 6
ERR_BREAKDOWN = 7
ERR_INVALID_CONFIG = 8
ERR_REACHED_END_TIME = 9
ERR_CUDA = 10
ERR_OUT_OF_MEMORY = 11
ERR_UNSUPPORTED = 12
ERR_INVALID_ARGUMENT = 13
ERR_TIMEOUT = 14

STATUS_NAMES = {
    0: "Ok", 1: "DimensionMismatch", 2: "InvalidCsr", 3: "IndexOutOfBounds", 4: "NonFiniteValue",
    5: "MissingDiagonal", 6: "ZeroDiagonal", 7: "Breakdown", 8: "InvalidConfig", 9: "ReachedEndTime",
    10: "Cuda", 11: "OutOfMemory", 12: "Unsupported", 13: "InvalidArgument", 14: "Timeout",
}

LINEAR_CONVERGED = 0
LINEAR_MAX_ITERATIONS = 1

CASE_CAVITY, CASE_CYLINDER, CASE_BACKWARD_STEP, CASE_CHANNEL = 0, 1, 2, 3
SIDE_LEFT, SIDE_RIGHT, SIDE_BOTTOM, SIDE_TOP = 0, 1, 2, 3
BOUNDARY_CASE_DEFAULT, BOUNDARY_VELOCITY, BOUNDARY_SYMMETRY, BOUNDARY_PRESSURE_OUTLET = 0, 1, 2, 3
CONVECTION_UPWIND, CONVECTION_CENTRAL = 0, 1
COUPLING_PROJECTION, COUPLING_SIMPLE = 0, 1
PRESSURE_PCG, PRESSURE_SOR, PRESSURE_FCG = 0, 1, 2
PRECISION_F64, PRECISION_MIXED = 0, 1
STOP_ABS_INF, STOP_REL_L2, STOP_REFERENCE_RESIDUAL = 0, 1, 2

FIELD_U, FIELD_V, FIELD_W, FIELD_PRESSURE, FIELD_RHS = 0, 1, 2, 3, 4
FIELD_U_STAR, FIELD_V_STAR, FIELD_W_STAR = 5, 6, 7
FIELD_SPEED, FIELD_VORTICITY, FIELD_U_CELL, FIELD_V_CELL = 8, 9, 10, 11
FIELD_TEMPERATURE = 12
SOLVE_GRAPH, SOLVE_RESIDENT, SOLVE_PERSISTENT, SOLVE_SOR, SOLVE_FCG = 0, 1, 2, 3, 4


class LinearSolverOptions(C.Structure):
    _fields_ = [
        ("absolute_tolerance", C.c_double),
        ("relative_tolerance", C.c_double),
        ("max_iterations", C.c_int64),
    ]


class LinearSolveReport(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("reserved", C.c_int32),
        ("iterations", C.c_int64),
        ("initial_residual", C.c_double),
        ("final_residual", C.c_double),
        ("relative_residual", C.c_double),
    ]


class CaseParams(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("reserved", C.c_int32),
        ("length", C.c_double),
        ("height", C.c_double),
        ("depth", C.c_double),
        ("density", C.c_double),
        ("kinematic_viscosity", C.c_double),
        ("reference_velocity", C.c_double),
        ("reynolds", C.c_double),
        ("cylinder_xc", C.c_double),
        ("cylinder_yc", C.c_double),
        ("cylinder_diameter", C.c_double),
        ("cylinder_perturbation", C.c_double),
        ("cylinder_mu", C.c_double),
        ("step_x", C.c_double),
        ("step_height", C.c_double),
    ]


class BoundaryOverride(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("reserved", C.c_int32),
        ("u", C.c_double),
        ("v", C.c_double),
        ("pressure", C.c_double),
    ]


ENERGY_OFF, ENERGY_CONSTANT_PROPERTIES = 0, 1
THERMAL_ADIABATIC, THERMAL_FIXED_TEMPERATURE = 0, 1
BUOYANCY_OFF, BUOYANCY_BOUSSINESQ = 0, 1


class ThermalBoundary(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("temperature", C.c_double)]


class PhysicsSettings(C.Structure):
    _fields_ = [
        ("energy_model", C.c_int32),
        ("buoyancy", C.c_int32),
        ("initial_temperature", C.c_double),
        ("thermal_diffusivity", C.c_double),
        ("source_temperature_rate", C.c_double),
        ("thermal", ThermalBoundary * 4),
        ("reference_temperature", C.c_double),
        ("thermal_expansion", C.c_double),
        ("gravity_x", C.c_double),
        ("gravity_y", C.c_double),
    ]


class CudaConfig(C.Structure):
    _fields_ = [
        ("abi_version", C.c_uint32),
        ("dimension", C.c_int32),
        ("case_params", CaseParams),
        ("overrides", BoundaryOverride * 4),
        ("nx", C.c_int64),
        ("ny", C.c_int64),
        ("nz", C.c_int64),
        ("dt", C.c_double),
        ("adaptive", C.c_int32),
        ("reserved0", C.c_int32),
        ("min_dt", C.c_double),
        ("max_dt", C.c_double),
        ("target_cfl", C.c_double),
        ("target_diffusion_number", C.c_double),
        ("max_growth_factor", C.c_double),
        ("max_steps", C.c_int64),
        ("t_end", C.c_double),
        ("convection", C.c_int32),
        ("coupling", C.c_int32),
        ("pressure_solver", C.c_int32),
        ("stop_rule", C.c_int32),
        ("pressure_max_iters", C.c_int64),
        ("pressure_tolerance", C.c_double),
        ("pressure_atol", C.c_double),
        ("pressure_rtol", C.c_double),
        ("pressure_omega", C.c_double),
        ("velocity_relaxation", C.c_double),
        ("pressure_relaxation", C.c_double),
        ("steady_tolerance", C.c_double),
        ("minimum_steps", C.c_int64),
        ("precision", C.c_int32),
        ("residual_replacement_every", C.c_int32),
        ("device", C.c_int32),
        ("reserved1", C.c_int32),
        ("fcg_weights_path", C.c_char_p),
        ("physics", PhysicsSettings),
    ]


class StepReport(C.Structure):
    _fields_ = [
        ("iteration", C.c_int64),
        ("time", C.c_double),
        ("time_step", C.c_double),
        ("continuity_residual", C.c_double),
        ("pressure_residual", C.c_double),
        ("pressure_iterations", C.c_int64),
        ("momentum_residual", C.c_double),
        ("max_speed", C.c_double),
        ("momentum_cfl", C.c_double),
        ("viscous_diffusion_number", C.c_double),
        ("drag_coefficient", C.c_double),
        ("lift_coefficient", C.c_double),
        ("converged", C.c_int32),
        ("reached_end_time", C.c_int32),
        ("pressure_initial_residual", C.c_double),
        ("pressure_true_relative_residual", C.c_double),
        ("pressure_solve_ms", C.c_double),
        ("step_ms", C.c_double),
        ("pressure_status", C.c_int32),
        ("fcg_fallback", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class BatchTuning(C.Structure):
    _fields_ = [
        ("tile_elems", C.c_int32 * 6),
        ("pressure_blocks_per_sm", C.c_int32),
        ("pressure_blocks", C.c_int32),
        ("graph_nodes", C.c_int32),
        ("reserved", C.c_int32),
        ("tune_ms", C.c_double),
    ]


class SimpleConfig(C.Structure):
    _fields_ = [
        ("abi_version", C.c_uint32),
        ("reserved", C.c_int32),
        ("nx", C.c_int64),
        ("ny", C.c_int64),
        ("length", C.c_double),
        ("height", C.c_double),
        ("kinematic_viscosity", C.c_double),
        ("inlet_peak_velocity", C.c_double),
        ("outlet_pressure", C.c_double),
        ("max_outer_iterations", C.c_int64),
        ("continuity_tolerance", C.c_double),
        ("velocity_relaxation", C.c_double),
        ("pressure_relaxation", C.c_double),
        ("momentum_solver", LinearSolverOptions),
        ("pressure_solver", LinearSolverOptions),
    ]


class SimpleReport(C.Structure):
    _fields_ = [
        ("converged", C.c_int32),
        ("reserved", C.c_int32),
        ("outer_iterations", C.c_int64),
        ("initial_continuity_rms", C.c_double),
        ("final_continuity_rms", C.c_double),
        ("momentum", LinearSolveReport * 3),
        ("pressure", LinearSolveReport),
        ("total_inflow", C.c_double),
        ("total_outflow", C.c_double),
        ("solve_ms", C.c_double),
    ]


BATCH_AUTOTUNE, BATCH_NO_GRAPH = 1, 2
FCG_LOSS_ENERGY, FCG_LOSS_RESIDUAL = 0, 1


class FcgReport(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("fallback", C.c_int32),
        ("fcg_iterations", C.c_int64),
        ("pcg_iterations", C.c_int64),
        ("initial_residual", C.c_double),
        ("final_residual", C.c_double),
        ("relative_residual", C.c_double),
        ("net_ms", C.c_double),
    ]

# Every extern "C" entry point of include/flursys_cuda.h: (restype, argtypes).
_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I64P = C.POINTER(C.c_int64)
SIGNATURES = {
    "flursys_cuda_abi_version": (C.c_uint32, []),
    "flursys_cuda_default_config": (C.c_int32, [C.c_int32, C.POINTER(CudaConfig)]),
    "flursys_cuda_create": (C.c_int32, [C.POINTER(CudaConfig), C.POINTER(_P)]),
    "flursys_cuda_step": (C.c_int32, [_P, C.c_int64, C.POINTER(StepReport)]),
    "flursys_cuda_download": (C.c_int32, [_P, C.c_int32, _D, C.c_size_t]),
    "flursys_cuda_upload": (C.c_int32, [_P, C.c_int32, _D, C.c_size_t]),
    "flursys_cuda_field_size": (C.c_size_t, [_P, C.c_int32]),
    "flursys_cuda_state": (C.c_int32, [_P, _I64P, _D]),
    "flursys_cuda_set_stream": (C.c_int32, [_P, _P]),
    "flursys_cuda_last_error": (C.c_int32, [_P, C.c_char_p, C.c_size_t]),
    "flursys_cuda_solver_profile": (C.c_int32, [_P, _D, C.c_size_t]),
    "flursys_cuda_destroy": (C.c_int32, [_P]),
    "flursys_cuda_global_error": (C.c_int32, [C.c_char_p, C.c_size_t]),
    "flursys_cuda_debug_inject_barrier_fault": (C.c_int32, [C.c_int32]),
    "flursys_cuda_snapshot_begin": (C.c_int32, [_P, C.POINTER(C.c_int32), C.c_int32, C.POINTER(_D),
                                                C.POINTER(C.c_size_t)]),
    "flursys_cuda_snapshot_wait": (C.c_int32, [_P]),
    "flursys_cuda_solve_kind": (C.c_int32, [_P, C.POINTER(C.c_int32)]),
    "flursys_cuda_csr_cg": (C.c_int32, [C.c_int64, C.c_int64, _I64P, _I64P, _D, _D, _D,
                                        C.POINTER(LinearSolverOptions), C.POINTER(LinearSolveReport)]),
    "flursys_cuda_csr_pcg": (C.c_int32, [C.c_int64, C.c_int64, _I64P, _I64P, _D, _D, _D,
                                         C.POINTER(LinearSolverOptions), C.POINTER(LinearSolveReport)]),
    "flursys_cuda_csr_bicgstab": (C.c_int32, [C.c_int64, C.c_int64, _I64P, _I64P, _D, _D, _D,
                                              C.POINTER(LinearSolverOptions), C.POINTER(LinearSolveReport)]),
    "flursys_cuda_csr_spmv": (C.c_int32, [C.c_int64, C.c_int64, C.c_int64, _I64P, _I64P, _D, _D, _D]),
    "flursys_cuda_stencil_pcg": (C.c_int32, [C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_double,
                                             C.c_double, _D, _D, C.c_int32,
                                             C.POINTER(LinearSolverOptions), C.POINTER(LinearSolveReport)]),
    # device pointers (rhs, x) and a cudaStream_t
    "flursys_cuda_stencil_pcg_noalloc": (C.c_int32, [C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_double,
                                                     C.c_double, _P, _P, C.c_int32,
                                                     C.POINTER(LinearSolverOptions), C.POINTER(LinearSolveReport),
                                                     _P]),
    "flursys_cuda_fcgnet_param_count": (C.c_int64, []),
    "flursys_cuda_fcgnet_create": (C.c_int32, [C.POINTER(C.c_float), C.POINTER(_P)]),
    "flursys_cuda_fcgnet_load": (C.c_int32, [C.c_char_p, C.POINTER(_P)]),
    "flursys_cuda_fcgnet_set_params": (C.c_int32, [_P, _P, _P]),
    "flursys_cuda_fcgnet_get_params": (C.c_int32, [_P, C.POINTER(C.c_float), C.c_int64]),
    "flursys_cuda_fcgnet_apply": (C.c_int32, [_P, C.c_int64, C.c_int64, C.c_int64, C.c_double, _P, _P, _P]),
    "flursys_cuda_fcgnet_train_sample": (C.c_int32, [_P, C.c_int64, C.c_int64, C.c_int64, _P, _P, C.c_double,
                                                     C.c_int32, _P, _P, _P]),
    "flursys_cuda_fcgnet_adam": (C.c_int32, [_P, _P, _P, _P, C.c_int64, C.c_float, C.c_float, C.c_float, C.c_float,
                                             C.c_int64, C.c_float, _P]),
    "flursys_cuda_fcgnet_destroy": (C.c_int32, [_P]),
    "flursys_cuda_stencil_fcg": (C.c_int32, [_P, C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_double,
                                             C.c_double, _D, _D, C.POINTER(LinearSolverOptions),
                                             C.POINTER(FcgReport)]),
    "flursys_cuda_simple_default_config": (C.c_int32, [C.POINTER(SimpleConfig)]),
    "flursys_cuda_simple_channel": (C.c_int32, [C.POINTER(SimpleConfig), _D, _D, _D, _D, _D,
                                                C.POINTER(SimpleReport)]),
    "flursys_cuda_batch_create": (C.c_int32, [C.POINTER(CudaConfig), C.c_int32, C.c_int32, C.POINTER(_P)]),
    "flursys_cuda_batch_step": (C.c_int32, [_P, C.c_int64]),
    "flursys_cuda_batch_report": (C.c_int32, [_P, C.c_int32, C.POINTER(StepReport), C.POINTER(C.c_int32)]),
    "flursys_cuda_batch_download": (C.c_int32, [_P, C.c_int32, C.c_int32, _D, C.c_size_t]),
    "flursys_cuda_batch_tuning": (C.c_int32, [_P, C.POINTER(BatchTuning)]),
    "flursys_cuda_batch_destroy": (C.c_int32, [_P]),
}

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libflursys_cuda.so")
_lib = None


def load() -> C.CDLL:
    """Loads libflursys_cuda.so (built in-tree) and binds every entry point."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m flursys_b200.build` "
            "(the CUDA backend has no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.flursys_cuda_abi_version() != ABI_VERSION:
        raise ImportError("libflursys_cuda.so ABI version does not match the Python binding")
    _lib = lib
    return lib


def dptr(a):
    """double* of a contiguous float64 numpy array."""
    return a.ctypes.data_as(_D)


def i64ptr(a):
    return a.ctypes.data_as(_I64P)
