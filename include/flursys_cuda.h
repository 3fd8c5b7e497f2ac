/*
 * flursys_cuda.h — C ABI of the B200 (sm_100a) backend for the FLURSYS
 * structured MAC projection step and its `src/linear` pressure solvers.
 *
 * Every entry point takes plain pointers and sizes, returns an int32 status
 * (FlursysStatus) and never aborts. Host pointers are borrowed for the
 * duration of a call only; a handle owns its device memory and one CUDA
 * stream. A handle is used by one host thread at a time; different handles
 * may run concurrently. Reference paths below are relative to the FLURSYS
 * source tree.
 */
#ifndef FLURSYS_CUDA_H
#define FLURSYS_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FLURSYS_CUDA_ABI_VERSION 2u

/* ------------------------------------------------------------------------
 * Status codes. 1..7 mirror LinearAlgebraError (src/linear/mod.rs:17-26);
 * the rest carry the solver-level `Err(String)` cases of
 * src/solver/incompressible.rs and src/solver/incompressible_3d.rs.
 * ---------------------------------------------------------------------- */
typedef enum FlursysStatus {
    FLURSYS_OK = 0,
    FLURSYS_ERR_DIMENSION_MISMATCH = 1,  /* LinearAlgebraError::DimensionMismatch */
    FLURSYS_ERR_INVALID_CSR = 2,         /* LinearAlgebraError::InvalidCsr */
    FLURSYS_ERR_INDEX_OUT_OF_BOUNDS = 3, /* LinearAlgebraError::IndexOutOfBounds */
    FLURSYS_ERR_NON_FINITE = 4,          /* LinearAlgebraError::NonFiniteValue, ensure_finite() */
    FLURSYS_ERR_MISSING_DIAGONAL = 5,    /* LinearAlgebraError::MissingDiagonal */
    FLURSYS_ERR_ZERO_DIAGONAL = 6,       /* LinearAlgebraError::ZeroDiagonal */
    FLURSYS_ERR_BREAKDOWN = 7,           /* LinearAlgebraError::Breakdown, PCG singular direction */
    FLURSYS_ERR_INVALID_CONFIG = 8,      /* SimulationConfig::validate, LidDrivenCavity3DConfig::validate */
    FLURSYS_ERR_REACHED_END_TIME = 9,    /* "projection simulation has already reached t_end" */
    FLURSYS_ERR_CUDA = 10,               /* a CUDA runtime call failed */
    FLURSYS_ERR_OUT_OF_MEMORY = 11,
    FLURSYS_ERR_UNSUPPORTED = 12,        /* a configuration this backend does not implement */
    FLURSYS_ERR_INVALID_ARGUMENT = 13,   /* null pointer, unknown enum value, wrong buffer size */
    FLURSYS_ERR_TIMEOUT = 14             /* a bounded device-side wait gave up */
} FlursysStatus;

/* LinearSolverStatus (src/linear/solver.rs:22-26). */
typedef enum FlursysLinearStatus {
    FLURSYS_LINEAR_CONVERGED = 0,
    FLURSYS_LINEAR_MAX_ITERATIONS = 1
} FlursysLinearStatus;

/* LinearSolverOptions (src/linear/solver.rs:5-20). Defaults: 1e-10, 1e-8, 1000. */
typedef struct FlursysLinearSolverOptions {
    double absolute_tolerance;
    double relative_tolerance;
    int64_t max_iterations;
} FlursysLinearSolverOptions;

/* LinearSolveReport (src/linear/solver.rs:28-35). */
typedef struct FlursysLinearSolveReport {
    int32_t status; /* FlursysLinearStatus */
    int32_t reserved;
    int64_t iterations;
    double initial_residual;
    double final_residual;
    double relative_residual;
} FlursysLinearSolveReport;

/* ------------------------------------------------------------------------
 * Case and solver configuration: a POD mirror of SimulationConfig
 * (src/solver/incompressible.rs:58-90) and LidDrivenCavity3DConfig
 * (src/solver/incompressible_3d.rs:8-25), plus backend knobs.
 * ---------------------------------------------------------------------- */
typedef enum FlursysCaseKind { /* CaseKind, src/cases/mod.rs:11-17 */
    FLURSYS_CASE_CAVITY = 0,
    FLURSYS_CASE_CYLINDER = 1,
    FLURSYS_CASE_BACKWARD_STEP = 2,
    FLURSYS_CASE_CHANNEL = 3
} FlursysCaseKind;

typedef enum FlursysSide { /* Side, src/cases/mod.rs:30-36 */
    FLURSYS_SIDE_LEFT = 0,
    FLURSYS_SIDE_RIGHT = 1,
    FLURSYS_SIDE_BOTTOM = 2,
    FLURSYS_SIDE_TOP = 3
} FlursysSide;

typedef enum FlursysBoundaryOverrideKind { /* SolverBoundaryOverride, src/preprocess.rs:1356-1361 */
    FLURSYS_BOUNDARY_CASE_DEFAULT = 0,
    FLURSYS_BOUNDARY_VELOCITY = 1,
    FLURSYS_BOUNDARY_SYMMETRY = 2,
    FLURSYS_BOUNDARY_PRESSURE_OUTLET = 3
} FlursysBoundaryOverrideKind;

typedef enum FlursysConvection { /* ConvectionScheme, src/solver/incompressible.rs:14-18 */
    FLURSYS_CONVECTION_UPWIND = 0,
    FLURSYS_CONVECTION_CENTRAL = 1
} FlursysConvection;

typedef enum FlursysCoupling { /* PressureVelocityCoupling, :26-33 */
    FLURSYS_COUPLING_PROJECTION = 0,
    FLURSYS_COUPLING_SIMPLE = 1
} FlursysCoupling;

typedef enum FlursysPressureSolver { /* PressureSolverKind, :20-24, plus the learned FCG */
    FLURSYS_PRESSURE_PCG = 0,
    FLURSYS_PRESSURE_SOR = 1, /* GPU: red-black ordering, not iterate-identical to the lexicographic sweep */
    FLURSYS_PRESSURE_FCG = 2  /* flexible CG with the learned preconditioner, Jacobi-PCG fallback */
} FlursysPressureSolver;

typedef enum FlursysPrecision {
    FLURSYS_PRECISION_F64 = 0,  /* every vector and reduction in FP64: parity mode */
    FLURSYS_PRECISION_MIXED = 1 /* FP32 stencil/SpMV vectors, FP64 dots, FP64 solution,
                                   FP64 residual replacement and final residual check */
} FlursysPrecision;

typedef enum FlursysStopRule {
    /* Reference 2D PCG: stop when max|r| < pressure_tolerance (incompressible.rs:1111-1115,1156-1164). */
    FLURSYS_STOP_ABS_INF = 0,
    /* src/linear convention: ||r||_2 <= pressure_atol + pressure_rtol * ||r0||_2 (solver.rs:84-85). */
    FLURSYS_STOP_REL_L2 = 1,
    /* Reference 3D SOR test: max|Lap(p) - rhs| over cells other than (0,0,0) < pressure_tolerance
       (incompressible_3d.rs:476-502). */
    FLURSYS_STOP_REFERENCE_RESIDUAL = 2
} FlursysStopRule;

typedef struct FlursysCaseParams { /* Case / CavityCase / ChannelCase / CylinderCase / BackwardStepCase */
    int32_t kind;                 /* FlursysCaseKind */
    int32_t reserved;
    double length, height, depth; /* domain extents; depth is used in 3D only */
    double density;
    double kinematic_viscosity;   /* 2D: Case::kinematic_viscosity(); 3D derives U*L/Re (incompressible_3d.rs:86-88) */
    double reference_velocity;    /* lid velocity, u_inf or u_mean */
    double reynolds;
    double cylinder_xc, cylinder_yc, cylinder_diameter, cylinder_perturbation, cylinder_mu;
    double step_x, step_height;
} FlursysCaseParams;

typedef struct FlursysBoundaryOverride {
    int32_t kind; /* FlursysBoundaryOverrideKind */
    int32_t reserved;
    double u, v;      /* Velocity override */
    double pressure;  /* PressureOutlet override */
} FlursysBoundaryOverride;

typedef enum FlursysEnergyModel { /* EnergyModel, src/physics.rs:9-15 */
    FLURSYS_ENERGY_OFF = 0,
    FLURSYS_ENERGY_CONSTANT_PROPERTIES = 1
} FlursysEnergyModel;

typedef enum FlursysThermalBoundaryKind { /* ThermalBoundaryCondition, src/physics.rs:17-25 */
    FLURSYS_THERMAL_ADIABATIC = 0,
    FLURSYS_THERMAL_FIXED_TEMPERATURE = 1
} FlursysThermalBoundaryKind;

typedef enum FlursysBuoyancyModel { /* BuoyancyModel, src/physics.rs:59-70 */
    FLURSYS_BUOYANCY_OFF = 0,
    FLURSYS_BUOYANCY_BOUSSINESQ = 1  /* body force g * beta * (T - T_ref) */
} FlursysBuoyancyModel;

typedef struct FlursysThermalBoundary {
    int32_t kind; /* FlursysThermalBoundaryKind */
    int32_t reserved;
    double temperature; /* FixedTemperature value */
} FlursysThermalBoundary;

/* PhysicsSettings (src/physics.rs:72-77): ThermalSettings (:27-56) and the
 * Boussinesq buoyancy parameters. 2D only: 3D configs with either model on
 * are rejected, as src/project.rs:276-284 rejects them. */
typedef struct FlursysPhysicsSettings {
    int32_t energy_model;           /* FlursysEnergyModel */
    int32_t buoyancy;               /* FlursysBuoyancyModel */
    double initial_temperature;     /* uniform initial temperature, K (default 293.15) */
    double thermal_diffusivity;     /* alpha = k / (rho cp), m^2/s (default 2.2e-5) */
    double source_temperature_rate; /* volumetric source as a temperature rate, K/s */
    FlursysThermalBoundary thermal[4]; /* indexed by FlursysSide */
    double reference_temperature;   /* Boussinesq T_ref */
    double thermal_expansion;       /* Boussinesq beta */
    double gravity_x, gravity_y;
} FlursysPhysicsSettings;

typedef struct FlursysCudaConfig {
    uint32_t abi_version; /* FLURSYS_CUDA_ABI_VERSION */
    int32_t dimension;    /* 2 or 3 */
    FlursysCaseParams case_params;
    FlursysBoundaryOverride overrides[4]; /* indexed by FlursysSide */
    int64_t nx, ny, nz;                   /* cells; nz ignored in 2D */
    double dt;
    /* TimeStepSettings (incompressible.rs:35-56) */
    int32_t adaptive;
    int32_t reserved0;
    double min_dt, max_dt, target_cfl, target_diffusion_number, max_growth_factor;
    int64_t max_steps;
    double t_end;
    int32_t convection;      /* FlursysConvection (3D always uses central advective form) */
    int32_t coupling;        /* FlursysCoupling (2D only) */
    int32_t pressure_solver; /* FlursysPressureSolver */
    int32_t stop_rule;       /* FlursysStopRule */
    int64_t pressure_max_iters;
    double pressure_tolerance;  /* ABS_INF and REFERENCE_RESIDUAL threshold */
    double pressure_atol;       /* REL_L2 absolute part */
    double pressure_rtol;       /* REL_L2 relative part */
    double pressure_omega;
    double velocity_relaxation, pressure_relaxation;
    double steady_tolerance;
    int64_t minimum_steps;
    /* backend knobs */
    int32_t precision;                  /* FlursysPrecision */
    int32_t residual_replacement_every; /* MIXED: FP64 true-residual replacement period (default 50) */
    int32_t device;                     /* CUDA ordinal */
    int32_t reserved1;
    const char *fcg_weights_path;       /* learned preconditioner weights (FCG only), may be NULL */
    FlursysPhysicsSettings physics;     /* SimulationConfig::physics (incompressible.rs:89) */
} FlursysCudaConfig;

/* SolverStep (incompressible.rs:211-229) plus backend diagnostics. */
typedef struct FlursysStepReport {
    int64_t iteration;
    double time;
    double time_step;
    double continuity_residual; /* max |div u| */
    double pressure_residual;   /* residual in the configured stop-rule norm */
    int64_t pressure_iterations;
    double momentum_residual;   /* max |u_new - u_old| over faces */
    double max_speed;
    double momentum_cfl;
    double viscous_diffusion_number;
    double drag_coefficient;
    double lift_coefficient;
    int32_t converged;
    int32_t reached_end_time;
    /* backend extras */
    double pressure_initial_residual;      /* ||r0|| in the stop-rule norm */
    double pressure_true_relative_residual; /* FP64 ||b - A x||_2 / ||r0||_2 after the solve */
    double pressure_solve_ms;              /* device time of the pressure solve (CUDA events) */
    double step_ms;                        /* device time of the whole step (CUDA events) */
    int32_t pressure_status;               /* FlursysLinearStatus */
    int32_t fcg_fallback;                  /* 1 when FCG stalled and Jacobi-PCG finished the solve */
} FlursysStepReport;

typedef enum FlursysFieldId {
    FLURSYS_FIELD_U = 0,        /* 2D (nx+1)*ny, 3D (nx+1)*ny*nz, x fastest */
    FLURSYS_FIELD_V = 1,        /* 2D nx*(ny+1), 3D nx*(ny+1)*nz */
    FLURSYS_FIELD_W = 2,        /* 3D nx*ny*(nz+1) */
    FLURSYS_FIELD_PRESSURE = 3, /* nx*ny(*nz) */
    FLURSYS_FIELD_RHS = 4,      /* pressure right-hand side of the last step */
    FLURSYS_FIELD_U_STAR = 5,
    FLURSYS_FIELD_V_STAR = 6,
    FLURSYS_FIELD_W_STAR = 7,
    FLURSYS_FIELD_SPEED = 8,    /* 2D cell-centred speed (compute_cell_fields, :1381-1439) */
    FLURSYS_FIELD_VORTICITY = 9,
    FLURSYS_FIELD_U_CELL = 10,
    FLURSYS_FIELD_V_CELL = 11,
    FLURSYS_FIELD_TEMPERATURE = 12 /* 2D cell temperature nx*ny, when the energy model is on */
} FlursysFieldId;

typedef struct FlursysCudaHandle FlursysCudaHandle;

/* Library ABI version (FLURSYS_CUDA_ABI_VERSION of the build). */
uint32_t flursys_cuda_abi_version(void);

/* Fills *cfg with the reference defaults: LidDrivenCavity3DConfig::default()
 * (incompressible_3d.rs:27-47) when dimension == 3, otherwise the CLI cavity
 * defaults of src/bin/flursys.rs:102-123,236-300. */
int32_t flursys_cuda_default_config(int32_t dimension, FlursysCudaConfig *cfg);

/* IncompressibleSolver::new (incompressible.rs:320-366) /
 * LidDrivenCavity3DSolver::new (incompressible_3d.rs:118-134): validates the
 * config, allocates device state, sets the initial field. */
int32_t flursys_cuda_create(const FlursysCudaConfig *cfg, FlursysCudaHandle **out);

/* Advances up to nsteps steps: advance_one_step (incompressible.rs:622-746,
 * incompressible_3d.rs:164-172). Stops early (2D) when the steady test of
 * run() (:478-485) passes or t_end is reached. `report` receives the last
 * step's SolverStep fields. */
int32_t flursys_cuda_step(FlursysCudaHandle *h, int64_t nsteps, FlursysStepReport *report);

/* Copies a device field to host memory (`n` doubles; must equal the field size). */
int32_t flursys_cuda_download(FlursysCudaHandle *h, int32_t field_id, double *host, size_t n);

/* Copies a host field to the device (parity inputs, restarts). */
int32_t flursys_cuda_upload(FlursysCudaHandle *h, int32_t field_id, const double *host, size_t n);

/* Element count of a field for this handle, or 0 if the field does not exist. */
size_t flursys_cuda_field_size(const FlursysCudaHandle *h, int32_t field_id);

/* Current step count and physical time. */
int32_t flursys_cuda_state(const FlursysCudaHandle *h, int64_t *step, double *time);

/* Makes the handle enqueue its work on `stream` (a cudaStream_t of the same
 * device; NULL restores the handle's own stream). Lets a caller time or
 * order the solver's kernels on a stream it owns. No reference counterpart:
 * the reference has no device streams. */
int32_t flursys_cuda_set_stream(FlursysCudaHandle *h, void *stream);

/* Device-time split of the last pressure solve of this handle, in ms:
 * [0] stencil passes, [1] pointwise passes, [2] grid barriers and partial
 * reductions, [3] FP64 residual replacements (as seen by block 0). For the
 * chip-resident 3D solve (FLURSYS_SOLVE_RESIDENT) the split is [0] face
 * exchange and direction update, [1] operator pass, [2] grid reductions and
 * barriers, [3] vector updates and residual replacements, [4] block 0's
 * waits inside grid barriers, [5] the largest [0] + [1] + [3] of any block
 * (the slowest block's work); the graph-driven 3D solve records none (all
 * zero). `n` is the capacity of `phase_ms` (up to 6 used). No reference
 * counterpart. */
int32_t flursys_cuda_solver_profile(const FlursysCudaHandle *h, double *phase_ms, size_t n);

/* Output overlapped with compute. No reference counterpart as an API: it
 * serves the snapshots that field_update() / prepare_output() take between
 * steps (incompressible.rs:563-586, output.rs:31-176) without stalling the
 * solver. snapshot_begin copies `count` fields (FlursysFieldId; each
 * host[i] holds sizes[i] doubles, ideally page-locked) into device snapshot
 * buffers on the handle's stream, ordered after the work already enqueued,
 * then drains them to the host buffers on a separate copy stream and
 * returns at once; steps called after it run while the copy drains.
 * snapshot_wait blocks until the host buffers hold the snapshot. One
 * snapshot may be pending per handle (FLURSYS_ERR_INVALID_ARGUMENT
 * otherwise); the host buffers must stay valid until snapshot_wait returns. */
int32_t flursys_cuda_snapshot_begin(FlursysCudaHandle *h, const int32_t *field_ids, int32_t count,
                                    double *const *host, const size_t *sizes);
int32_t flursys_cuda_snapshot_wait(FlursysCudaHandle *h);

/* Which implementation runs the pressure solve of a 3D handle (diagnostic;
 * no reference counterpart): FlursysSolveKind. */
typedef enum FlursysSolveKind {
    FLURSYS_SOLVE_GRAPH = 0,      /* PCG as a kernel sequence in one CUDA graph (2 kernels per iteration) */
    FLURSYS_SOLVE_RESIDENT = 1,   /* PCG as one cooperative launch with its state on the chip */
    FLURSYS_SOLVE_PERSISTENT = 2, /* PCG as one cooperative launch streaming its vectors */
    FLURSYS_SOLVE_SOR = 3,        /* red-black SOR */
    FLURSYS_SOLVE_FCG = 4         /* learned-preconditioner flexible CG */
} FlursysSolveKind;
int32_t flursys_cuda_solve_kind(const FlursysCudaHandle *h, int32_t *kind);

/* Copies the last error message (NUL-terminated, truncated to `size`). */
int32_t flursys_cuda_last_error(const FlursysCudaHandle *h, char *buf, size_t size);

/* Releases device memory and the stream. */
int32_t flursys_cuda_destroy(FlursysCudaHandle *h);

/* Message for the last failed call on this thread that had no handle. */
int32_t flursys_cuda_global_error(char *buf, size_t size);

/* Host-side fault injection for tests of the bounded device waits. No
 * reference counterpart. The next persistent 3D PCG launch (the kernel of
 * flursys_cuda_stencil_pcg with nz >= 2, of flursys_cuda_stencil_pcg_noalloc,
 * of 3D handles configured with the persistent solver, and the chip-resident
 * MIXED solve of 3D handles) waits at its grid
 * barriers for `extra_arrivals` blocks that were never launched, with a poll
 * limit of a few milliseconds; every wait gives up, the kernel returns, and
 * the call reports FLURSYS_ERR_TIMEOUT with the device context intact. The
 * injection applies to one launch and is then cleared; 0 cancels a pending
 * one. Returns FLURSYS_ERR_INVALID_ARGUMENT for a negative count. */
int32_t flursys_cuda_debug_inject_barrier_fault(int32_t extra_arrivals);

/* ------------------------------------------------------------------------
 * Linear solvers with the src/linear signatures (src/linear/solver.rs:43-60,
 * 155-160). CSR arrays are host memory with int64 offsets/columns; `x_inout`
 * carries the initial guess in and the solution out. Status mirrors
 * LinearAlgebraError. All arithmetic is FP64 on the device.
 * ---------------------------------------------------------------------- */
int32_t flursys_cuda_csr_cg(int64_t n, int64_t nnz, const int64_t *row_offsets,
                            const int64_t *columns, const double *values, const double *rhs,
                            double *x_inout, const FlursysLinearSolverOptions *options,
                            FlursysLinearSolveReport *report);
int32_t flursys_cuda_csr_pcg(int64_t n, int64_t nnz, const int64_t *row_offsets,
                             const int64_t *columns, const double *values, const double *rhs,
                             double *x_inout, const FlursysLinearSolverOptions *options,
                             FlursysLinearSolveReport *report);
int32_t flursys_cuda_csr_bicgstab(int64_t n, int64_t nnz, const int64_t *row_offsets,
                                  const int64_t *columns, const double *values, const double *rhs,
                                  double *x_inout, const FlursysLinearSolverOptions *options,
                                  FlursysLinearSolveReport *report);

/* CsrMatrix::spmv_into (src/linear/csr.rs:89-106) on the device. */
int32_t flursys_cuda_csr_spmv(int64_t nrows, int64_t ncols, int64_t nnz,
                              const int64_t *row_offsets, const int64_t *columns,
                              const double *values, const double *input, double *output);

/* Matrix-free pressure PCG on a structured grid: the operator of
 * apply_pressure_operator (incompressible.rs:1216-1255) in 2D (nz == 1) or the
 * pinned 7-point Neumann operator of incompressible_3d.rs:293-332 in 3D.
 * `rhs` is the Poisson right-hand side (as built by build_pressure_rhs);
 * the solved system is A x = -rhs with A the positive operator. */
int32_t flursys_cuda_stencil_pcg(int64_t nx, int64_t ny, int64_t nz, double dx, double dy,
                                 double dz, const double *rhs, double *x_inout,
                                 int32_t precision, const FlursysLinearSolverOptions *options,
                                 FlursysLinearSolveReport *report);

/* Allocation-free variant of the 3D matrix-free pressure PCG. No reference
 * counterpart: the reference solves on the host and has no device memory.
 *
 * Some callers cannot let a library allocate device memory: applications
 * whose device memory is entirely owned by their own pool allocator (a
 * cudaMalloc would fail or fragment it), services running under a hard
 * per-process memory cap, and latency-sensitive pipelines that cannot take
 * the device-wide synchronisation a cudaFree implies. This entry point calls
 * no cudaMalloc, cudaFree or other allocating routine: it solves the same
 * pinned 7-point system as flursys_cuda_stencil_pcg (nz >= 2; A x = -rhs,
 * x(0,0,0) = 0; stop when ||r||_2 <= atol + rtol ||r0||_2) with the same
 * kernel, on caller-owned DEVICE buffers `rhs_device` and `x_device`
 * (nx*ny*nz FP64 values each, 16-byte aligned; x_device holds the initial
 * guess in and the solution out), enqueued on `stream` (NULL = the default
 * stream); it returns after the solve, with `report` filled.
 *
 * Its scratch (work vectors, partial sums, barrier, result) is one
 * file-scope device array of about 9.2 MB that every device loading the
 * library keeps until the process exits. Limit: nx*ny*nz <= 262144 cells
 * (64^3); larger grids are rejected with FLURSYS_ERR_INVALID_ARGUMENT and a
 * message in flursys_cuda_global_error(). Every call shares the array and
 * it keeps the last call's contents, so calls that overlap on the GPU (two
 * host threads, two streams) race; run them one after another. The first
 * call on a device looks up the array's device address with that device
 * current; make that first call before any stream capture. */
int32_t flursys_cuda_stencil_pcg_noalloc(int64_t nx, int64_t ny, int64_t nz, double dx, double dy, double dz,
                                         const double *rhs_device, double *x_device, int32_t precision,
                                         const FlursysLinearSolverOptions *options,
                                         FlursysLinearSolveReport *report, void *stream);

/* ---- Learned preconditioner and flexible CG (3D pinned pressure system) ----
 * No reference counterpart: the reference's pressure solvers are SOR and
 * Jacobi-PCG (src/linear/solver.rs, src/solver/incompressible_3d.rs:293-332).
 * The network is a linear 4-level 3x3x3 convolutional encoder-decoder
 * (channels 16/32/64/64, BF16 activations, FP32 accumulation) applied to
 * the residual; its FP32 parameters are laid out layer after layer as
 * W[co][tap][ci] (flursys_cuda_fcgnet_param_count() floats). Grids must have
 * nx, ny, nz divisible by 8. Every buffer argument named *_device is device
 * memory; `stream` is a cudaStream_t (NULL = default stream). */
typedef struct FlursysFcgNet FlursysFcgNet;

typedef struct FlursysFcgReport {
    int32_t status;           /* FlursysLinearStatus of the whole solve */
    int32_t fallback;         /* 1 when the Jacobi-PCG fallback finished the solve */
    int64_t fcg_iterations;
    int64_t pcg_iterations;   /* fallback iterations */
    double initial_residual;  /* ||b - A x0||_2 */
    double final_residual;    /* FP64 ||b - A x||_2 of the returned solution */
    double relative_residual;
    double net_ms;            /* device time spent applying the network */
} FlursysFcgReport;

int64_t flursys_cuda_fcgnet_param_count(void);
/* params: host FP32 parameters, or NULL for zeros. */
int32_t flursys_cuda_fcgnet_create(const float *params, FlursysFcgNet **out);
/* Weights file: "FLNT", uint32 version 1, uint32 layer count 7, (cin, cout)
 * int32 pairs, int64 parameter count, FP32 parameters, little endian. */
int32_t flursys_cuda_fcgnet_load(const char *path, FlursysFcgNet **out);
int32_t flursys_cuda_fcgnet_set_params(FlursysFcgNet *net, const float *params_device, void *stream);
int32_t flursys_cuda_fcgnet_get_params(const FlursysFcgNet *net, float *host, int64_t count);
/* z = M(r) on an nx*ny*nz grid with cell spacing factor h2 (h^2 of A^-1). */
int32_t flursys_cuda_fcgnet_apply(FlursysFcgNet *net, int64_t nx, int64_t ny, int64_t nz, double h2,
                                  const float *r_device, float *z_device, void *stream);
/* Training losses of e = net(b_hat) - p_hat on the unit-spacing pure-Neumann
 * 7-point operator L (out-of-range neighbours dropped), with L p_hat = b_hat
 * and sum(b_hat) = 0 (the FCG solves the pinned system in this compatible
 * Neumann form):
 *   ENERGY    (e . L e) / norm, norm = p_hat . b_hat
 *   RESIDUAL  |L e|^2 / norm,   norm = b_hat . b_hat  (= |L net(b_hat) - b_hat|^2 / |b_hat|^2) */
enum FlursysFcgLoss { FLURSYS_FCG_LOSS_ENERGY = 0, FLURSYS_FCG_LOSS_RESIDUAL = 1 };
/* One training sample: forward on b_hat, loss, backward; adds dLoss/dparams
 * into grad_device and the loss into *loss_device (one double). */
int32_t flursys_cuda_fcgnet_train_sample(FlursysFcgNet *net, int64_t nx, int64_t ny, int64_t nz,
                                         const float *b_hat_device, const float *p_hat_device, double norm,
                                         int32_t loss_kind, float *grad_device, double *loss_device, void *stream);
/* Adam step on FP32 parameters (bias-corrected, step t >= 1). */
int32_t flursys_cuda_fcgnet_adam(float *params_device, const float *grad_device, float *m_device, float *v_device,
                                 int64_t n, float lr, float beta1, float beta2, float eps, int64_t t,
                                 float grad_scale, void *stream);
int32_t flursys_cuda_fcgnet_destroy(FlursysFcgNet *net);
/* Learned-preconditioner FCG on the pinned 3D system of
 * flursys_cuda_stencil_pcg (host buffers): stops when ||b - A x||_2 <= atol
 * + rtol ||b - A x0||_2 (FP64), Jacobi-PCG finishing the solve when FCG
 * stalls. options->max_iterations caps the FCG iterations. */
int32_t flursys_cuda_stencil_fcg(FlursysFcgNet *net, int64_t nx, int64_t ny, int64_t nz, double dx, double dy,
                                 double dz, const double *rhs, double *x_inout,
                                 const FlursysLinearSolverOptions *options, FlursysFcgReport *report);

/* ---- Steady collocated SIMPLE channel -------------------------------------
 * solve_incompressible (src/unstructured_incompressible.rs:368-482) with
 * solve_simple (src/simple.rs:148-314) on a plane channel of nx x ny uniform
 * quads (unit depth): inlet on the left (fixed velocity), no-slip walls at
 * the bottom and top, pressure outlet on the right. Kinematic pressure (the
 * SIMPLE core uses unit density). Each outer iteration assembles the
 * momentum systems to CSR and solves them with BiCGSTAB, forms the
 * Rhie-Chow face flux, assembles the pressure-correction system to CSR and
 * solves it with Jacobi-PCG, and corrects pressure, velocity and face flux;
 * it stops when the RMS of the integrated cell continuity imbalance is at
 * most continuity_tolerance. The inlet profile is parabolic, u = peak 4 y
 * (H - y) / H^2 at each face centre: a per-face fixed velocity where the
 * reference's VelocityInlet holds one vector per patch. */
typedef struct FlursysSimpleConfig {
    uint32_t abi_version;
    int32_t reserved;
    int64_t nx, ny;
    double length, height;
    double kinematic_viscosity;
    double inlet_peak_velocity;
    double outlet_pressure;
    int64_t max_outer_iterations;          /* IncompressibleSolverOptions defaults: 200 */
    double continuity_tolerance;           /* 1e-10 */
    double velocity_relaxation;            /* 0.7 */
    double pressure_relaxation;            /* 0.3 */
    FlursysLinearSolverOptions momentum_solver;  /* LinearSolverOptions::default() */
    FlursysLinearSolverOptions pressure_solver;
} FlursysSimpleConfig;

typedef struct FlursysSimpleReport {     /* IncompressibleSolveReport / SimpleReport */
    int32_t converged;
    int32_t reserved;
    int64_t outer_iterations;
    double initial_continuity_rms;
    double final_continuity_rms;
    FlursysLinearSolveReport momentum[3];  /* x, y, z systems of the last outer iteration */
    FlursysLinearSolveReport pressure;     /* pressure correction of the last outer iteration */
    double total_inflow, total_outflow;    /* boundary flux sums (inflow negative) */
    double solve_ms;                       /* device time of the whole solve */
} FlursysSimpleReport;

int32_t flursys_cuda_simple_default_config(FlursysSimpleConfig *cfg);
/* Host outputs (any may be NULL): cell velocity components and pressure
 * (nx*ny, x fastest), face fluxes ((nx+1)*ny x-faces then nx*(ny+1)
 * y-faces, each positive along +x / +y), and the continuity RMS history
 * (max_outer_iterations + 1 values: the initial one, then one per outer
 * iteration). Errors mirror SimpleError: a linear solve that does not
 * converge is FLURSYS_ERR_BREAKDOWN with the message naming it. */
int32_t flursys_cuda_simple_channel(const FlursysSimpleConfig *cfg, double *velocity_x, double *velocity_y,
                                    double *pressure, double *face_flux, double *continuity_history,
                                    FlursysSimpleReport *report);

/* ---- Batched 2D solvers ---------------------------------------------------
 * Many independent 2D projection solvers (one IncompressibleSolver,
 * src/solver/incompressible.rs:294-746, per config) of uneven size advanced
 * together on one device. No reference counterpart: the reference runs one
 * solver per process; each instance here computes what that solver computes.
 *
 * Every config must be 2D, projection coupling, pressure solver PCG or SOR,
 * and all configs must share one `precision`. Each instance keeps its own
 * dt control (fixed dt, or adaptive_time_step :2308-2336), its own t_end and
 * its own pressure-solver settings. One step of the batch is one captured
 * CUDA graph: per instance the dt rule, momentum predictor, boundaries,
 * pressure right-hand side, pressure solve (one cooperative launch over all
 * instances, blocks shared out in proportion to cells x iterations of the
 * previous step), correction and diagnostics. An instance that reaches t_end
 * or fails stops stepping; the others go on. */
typedef struct FlursysBatchHandle FlursysBatchHandle;

enum FlursysBatchFlags {
    FLURSYS_BATCH_AUTOTUNE = 1, /* time candidate tile sizes and pressure grids at create */
    FLURSYS_BATCH_NO_GRAPH = 2  /* enqueue the kernels of each step directly (no graph) */
};

/* Tuned launch parameters (flursys_cuda_batch_tuning). */
typedef struct FlursysBatchTuning {
    int32_t tile_elems[6];      /* elements per tile: predict, boundaries, rhs, correct, boundaries, post */
    int32_t pressure_blocks_per_sm;
    int32_t pressure_blocks;    /* blocks of the cooperative pressure launch */
    int32_t graph_nodes;        /* kernel nodes of one step's graph (0 without a graph) */
    int32_t reserved;
    double tune_ms;             /* host time spent tuning at create */
} FlursysBatchTuning;

int32_t flursys_cuda_batch_create(const FlursysCudaConfig *configs, int32_t count, int32_t flags,
                                  FlursysBatchHandle **out);
/* Advances every active instance by `nsteps` steps (instances that stop
 * early stay put) and returns after the last one. FLURSYS_OK unless the
 * device failed (FLURSYS_ERR_CUDA, FLURSYS_ERR_TIMEOUT); per-instance
 * outcomes come from flursys_cuda_batch_report. */
int32_t flursys_cuda_batch_step(FlursysBatchHandle *h, int64_t nsteps);
/* Report of the last step `instance` took (SolverStep, :211-229) and its
 * status: FLURSYS_OK while it steps, FLURSYS_ERR_REACHED_END_TIME once its
 * time reached t_end, or the error that stopped it. step_ms is the mean
 * device time of one batch step over the last flursys_cuda_batch_step call;
 * pressure_solve_ms is 0 (the solve is shared by all instances). */
int32_t flursys_cuda_batch_report(FlursysBatchHandle *h, int32_t instance, FlursysStepReport *report,
                                  int32_t *instance_status);
/* Copies field `field_id` (FlursysFieldId, 2D fields) of one instance. */
int32_t flursys_cuda_batch_download(FlursysBatchHandle *h, int32_t instance, int32_t field_id, double *host,
                                    size_t n);
int32_t flursys_cuda_batch_tuning(const FlursysBatchHandle *h, FlursysBatchTuning *out);
int32_t flursys_cuda_batch_destroy(FlursysBatchHandle *h);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* FLURSYS_CUDA_H */
