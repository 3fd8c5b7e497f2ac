// capi_internal.cuh — the handle behind FlursysCudaHandle and the helpers
// shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "cavity3d.cuh"
#include "common.cuh"
#include "flursys_cuda.h"
#include "pcg3d.cuh"
#include "pcg3d_seq.cuh"

namespace flursys {

// Device work vectors of one structured PCG solve (sized for n cells).
struct PcgWorkspace {
    int grid = 0;
    void *r = nullptr, *d0 = nullptr, *d1 = nullptr, *q = nullptr;
    void *r_z = nullptr;  // 2D: stored preconditioned residual
    float *dx = nullptr;
    double *partials = nullptr;
    GridBarrier *barrier = nullptr;
    PcgResultDev *result = nullptr;
    PcgResultDev *h_result = nullptr;  // pinned host copy
    unsigned char *row_class = nullptr;  // 3D: per-row boundary class
    int precision = 0;
    cudaError_t allocate(long long n, int precision, int device, int dim);
    // 3D pressure solves also need the per-row boundary class table.
    cudaError_t allocate3d(int nx, int ny, int nz, int precision, int device, cudaStream_t stream);
    void free_all();
};

struct Handle2D;

}  // namespace flursys

struct FlursysCudaHandle {
    FlursysCudaConfig cfg{};
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    std::string err;
    int64_t step = 0;
    double time = 0.0;
    // 3D state
    flursys::Cavity3dState s3{};
    flursys::Diag3Dev *diag3 = nullptr;
    flursys::Diag3Dev *h_diag3 = nullptr;
    flursys::PcgWorkspace pcg;
    flursys::Pcg3dSeqPlan seq;   // graph-driven PCG (default 3D PCG path)
    bool use_seq = false;
    flursys::CgSeqState *h_seq = nullptr;  // pinned host copy of the solve state
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    // 2D state
    flursys::Handle2D *h2 = nullptr;
    // 3D learned-preconditioner FCG (pressure_solver == FLURSYS_PRESSURE_FCG)
    FlursysFcgNet *fcg_net = nullptr;
    FlursysFcgReport fcg_report{};
    // asynchronous snapshots: device copies of the fields, drained to the
    // caller's host buffers on a copy stream while later steps run
    double *snap_buf[16] = {};
    size_t snap_n[16] = {};
    cudaStream_t snap_stream = nullptr;
    cudaEvent_t snap_taken = nullptr, snap_done = nullptr;
    bool snap_pending = false;
};

namespace flursys {

int32_t set_cuda_error(std::string *dst, cudaError_t e, const char *what);
// Rust's `{:.Ne}` rendering of an f64 ("1.500e-5"), for messages that
// callers compare with the reference's.
std::string rust_sci(double v, int prec);
// ensure_finite's message for the non-finite value at `index` of the device
// array `field`: "Non-finite {name} value at flat index {i}: {v} (step {s})"
// in 2D (incompressible.rs:1707-1742), "Non-finite 3D {name} value at flat
// index {i}: {v}" in 3D (incompressible_3d.rs:534-554).
std::string nonfinite_message(const char *name, unsigned long long index, const double *field, long long step,
                              bool two_d);
// SimulationConfig::validate / LidDrivenCavity3DConfig::validate of a config.
int32_t validate_config_checked(const FlursysCudaConfig &c, std::string *msg);
// Message returned by flursys_cuda_global_error() on this thread.
void set_global_error(const std::string &msg);
// Matrix-free 2D pressure PCG for flursys_cuda_stencil_pcg (nz == 1).
int32_t stencil_pcg2d(int64_t nx, int64_t ny, double dx, double dy, const double *rhs, double *x_inout,
                      int32_t precision, const FlursysLinearSolverOptions *options,
                      FlursysLinearSolveReport *report);
int32_t handle_init(FlursysCudaHandle *h, const FlursysCudaConfig *cfg);
void handle_free(FlursysCudaHandle *h);
int32_t step3d(FlursysCudaHandle *h, FlursysStepReport *rep);
int32_t step2d(FlursysCudaHandle *h, FlursysStepReport *rep);
bool field_ptr(FlursysCudaHandle *h, int32_t id, double **p, size_t *n);
void on_upload2d(FlursysCudaHandle *h, int32_t id);
int32_t init2d(FlursysCudaHandle *h);
void free2d(FlursysCudaHandle *h);
bool field_ptr2d(FlursysCudaHandle *h, int32_t id, double **p, size_t *n);

// Host-side data of one 2D case (src/cases/mod.rs:120-227 with the
// SolverBoundaryOverrides of src/preprocess.rs:1370-1388): boundary kinds,
// cell flags, boundary velocity arrays and the initial field of
// initialize_velocity (incompressible.rs:588-620).
struct Case2dHost {
    int kind[4];          // BoundaryKindDev per side
    double outlet_p;      // right-side outlet pressure
    bool project;         // pure Neumann pressure system (no outlet)
    std::vector<uint8_t> flags;  // CellFlag bits, nx*ny
    long long fluid;      // cells that are neither solid nor outlet
    int ref_cell;         // first non-solid cell
    // bu_left, bu_right, bv_bottom, bv_top, gu_bottom, gu_top, gv_left, gv_right
    std::vector<double> bnd[8];
    std::vector<double> u, v;    // initial face velocities
    double max_u, max_v;  // max |u|, |v| of the initial field
};
void build_case2d(const FlursysCudaConfig &c, Case2dHost *out);
int32_t run_pcg3d(PcgWorkspace &ws, int nx, int ny, int nz, double dx, double dy, double dz, double *x,
                  const double *rhs, int precision, int stop_rule, double tol, double atol, double rtol,
                  long long max_iters, int replace_every, cudaStream_t stream, std::string *err);
// Maps a finished PcgResultDev to a status and message.
int32_t pcg_result_status(const PcgResultDev &r, std::string *err);
// Learned-preconditioner FCG on device buffers x (FP64, in/out) and rhs
// (A x = -rhs on the pinned 3D system); fallback Jacobi-PCG in
// `precision_fallback`.
int32_t fcg_solve(FlursysFcgNet *net, int nx, int ny, int nz, double dx, double dy, double dz, double *x,
                  const double *rhs, double atol, double rtol, long long max_iters, int precision_fallback,
                  cudaStream_t st, FlursysFcgReport *rep, std::string *err);
int32_t fcgnet_read_file(const char *path, std::vector<float> *out, std::string *err);
int32_t fcgnet_create(const float *host_params, FlursysFcgNet **out, std::string *err);
void fcgnet_destroy(FlursysFcgNet *net);
// Fills the argument block of a 3D pressure solve on the workspace buffers.
Pcg3dArgs make_pcg3d_args(PcgWorkspace &ws, int nx, int ny, int nz, double dx, double dy, double dz, double *x,
                          const double *rhs, int precision, int stop_rule, double tol, double atol, double rtol,
                          long long max_iters, int replace_every);

}  // namespace flursys
