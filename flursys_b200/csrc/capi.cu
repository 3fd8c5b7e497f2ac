// capi.cu — the extern "C" boundary of libflursys_cuda.so (include/flursys_cuda.h).
//
// Host-side mirror of the reference solver objects: a FlursysCudaHandle plays
// the role of IncompressibleSolver (src/solver/incompressible.rs:294-317) or
// LidDrivenCavity3DSolver (src/solver/incompressible_3d.rs:103-115). It owns
// device memory and one stream; every call validates its arguments, returns
// a FlursysStatus and keeps a message for flursys_cuda_last_error().
#include <cuda_runtime.h>

#include <atomic>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "capi_internal.cuh"
#include "cavity2d.cuh"
#include "cavity3d.cuh"
#include "common.cuh"
#include "csr.cuh"
#include "flursys_cuda.h"
#include "pcg2d.cuh"
#include "pcg3d.cuh"

using namespace flursys;

namespace {

thread_local std::string g_error;

void copy_msg(const std::string &s, char *buf, size_t size) {
    if (!buf || size == 0) return;
    size_t n = std::min(size - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = '\0';
}

// SimulationConfig::validate (incompressible.rs:93-191, with
// PhysicsSettings::validate, src/physics.rs:79-131) and
// LidDrivenCavity3DConfig::validate (incompressible_3d.rs:50-84).
int32_t validate_config(const FlursysCudaConfig &c, std::string *msg) {
    auto fin_pos = [](double x) { return std::isfinite(x) && x > 0.0; };
    if (c.abi_version != FLURSYS_CUDA_ABI_VERSION) { *msg = "config abi_version does not match the library"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    if (c.precision != FLURSYS_PRECISION_F64 && c.precision != FLURSYS_PRECISION_MIXED) { *msg = "unknown precision"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    if (c.stop_rule < FLURSYS_STOP_ABS_INF || c.stop_rule > FLURSYS_STOP_REFERENCE_RESIDUAL) { *msg = "unknown stop rule"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    if (c.pressure_solver < FLURSYS_PRESSURE_PCG || c.pressure_solver > FLURSYS_PRESSURE_FCG) { *msg = "unknown pressure solver"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    if (c.stop_rule == FLURSYS_STOP_REL_L2 &&
        !(std::isfinite(c.pressure_atol) && c.pressure_atol >= 0.0 && std::isfinite(c.pressure_rtol) && c.pressure_rtol >= 0.0)) {
        *msg = "pressure_atol and pressure_rtol must be finite and non-negative";
        return FLURSYS_ERR_INVALID_CONFIG;
    }
    if (c.precision == FLURSYS_PRECISION_MIXED && c.residual_replacement_every < 1) { *msg = "residual_replacement_every must be positive"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (c.dimension == 3) {
        if (c.case_params.kind != FLURSYS_CASE_CAVITY) { *msg = "the current 3D backend supports only a lid-driven cavity case"; return FLURSYS_ERR_UNSUPPORTED; }
        // src/project.rs:276-284: the 3D backend runs constant-property flow only
        if (c.physics.energy_model != FLURSYS_ENERGY_OFF || c.physics.buoyancy != FLURSYS_BUOYANCY_OFF) { *msg = "the current 3D backend supports constant-property flow only; thermal and buoyancy models are not available"; return FLURSYS_ERR_UNSUPPORTED; }
        if (c.nx < 4 || c.ny < 4 || c.nz < 4) { *msg = "nx, ny, and nz must all be at least 4"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!(c.case_params.length > 0.0 && c.case_params.height > 0.0 && c.case_params.depth > 0.0)) { *msg = "Domain dimensions must be positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!fin_pos(c.case_params.density)) { *msg = "density must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!fin_pos(c.case_params.reference_velocity)) { *msg = "lid_velocity must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!fin_pos(c.case_params.reynolds)) { *msg = "reynolds must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!fin_pos(c.dt)) { *msg = "dt must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (c.max_steps <= 0 || c.pressure_max_iters <= 0) { *msg = "iteration limits must be positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!fin_pos(c.pressure_tolerance)) { *msg = "pressure_tolerance must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!(std::isfinite(c.pressure_omega) && c.pressure_omega > 0.0 && c.pressure_omega < 2.0)) { *msg = "pressure_omega must lie between 0 and 2"; return FLURSYS_ERR_INVALID_CONFIG; }
        // Device indices are 32-bit: the face arrays must stay below 2^31 entries.
        if (c.nx > (1 << 20) || c.ny > (1 << 20) || c.nz > (1 << 20) ||
            (c.nx + 1) * (c.ny + 1) * (c.nz + 1) >= (1LL << 31)) { *msg = "grid too large for this backend"; return FLURSYS_ERR_INVALID_CONFIG; }
        return FLURSYS_OK;
    }
    if (c.dimension != 2) { *msg = "dimension must be 2 or 3"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    if (c.pressure_solver == FLURSYS_PRESSURE_FCG) { *msg = "the learned FCG pressure solver is 3D only"; return FLURSYS_ERR_UNSUPPORTED; }
    if (c.case_params.kind < FLURSYS_CASE_CAVITY || c.case_params.kind > FLURSYS_CASE_CHANNEL) { *msg = "unknown case kind"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    for (int s = 0; s < 4; ++s)
        if (c.overrides[s].kind < FLURSYS_BOUNDARY_CASE_DEFAULT || c.overrides[s].kind > FLURSYS_BOUNDARY_PRESSURE_OUTLET) { *msg = "unknown boundary override kind"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    if (c.nx < 4 || c.ny < 4) { *msg = "nx and ny must be at least 4"; return FLURSYS_ERR_INVALID_CONFIG; }
    // Device indices are 32-bit: the face arrays must stay below 2^31 entries.
    if (c.nx > (1 << 20) || c.ny > (1 << 20) || (c.nx + 1) * (c.ny + 1) >= (1LL << 31)) { *msg = "grid dimension too large"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (!fin_pos(c.dt)) { *msg = "dt must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (!std::isfinite(c.t_end) || c.t_end < 0.0) { *msg = "t_end must be finite and non-negative"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (c.coupling == FLURSYS_COUPLING_PROJECTION && c.t_end == 0.0) { *msg = "t_end must be positive for projection coupling"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (c.max_steps <= 0) { *msg = "max_steps must be positive"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (c.pressure_max_iters <= 0) { *msg = "pressure_max_iters must be positive"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (!std::isfinite(c.pressure_omega) || c.pressure_omega <= 0.0 || c.pressure_omega >= 2.0) { *msg = "pressure_omega must lie between 0 and 2"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (!std::isfinite(c.velocity_relaxation) || c.velocity_relaxation <= 0.0 || c.velocity_relaxation > 1.0) { *msg = "velocity_relaxation must lie between 0 (exclusive) and 1"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (!std::isfinite(c.pressure_relaxation) || c.pressure_relaxation <= 0.0 || c.pressure_relaxation > 1.0) { *msg = "pressure_relaxation must lie between 0 (exclusive) and 1"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (!fin_pos(c.steady_tolerance)) { *msg = "steady_tolerance must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (!fin_pos(c.case_params.density) || !fin_pos(c.case_params.kinematic_viscosity)) { *msg = "fluid density and kinematic viscosity must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (c.adaptive) {
        if (c.coupling != FLURSYS_COUPLING_PROJECTION) { *msg = "adaptive time stepping requires transient projection coupling"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!fin_pos(c.min_dt)) { *msg = "adaptive min_dt must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!fin_pos(c.max_dt)) { *msg = "adaptive max_dt must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (c.min_dt > c.max_dt) { *msg = "adaptive min_dt must not exceed max_dt"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (c.dt < c.min_dt || c.dt > c.max_dt) { *msg = "adaptive initial dt must lie between min_dt and max_dt"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!std::isfinite(c.target_cfl) || c.target_cfl <= 0.0 || c.target_cfl > 1.0) { *msg = "adaptive target_cfl must lie between 0 (exclusive) and 1"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!std::isfinite(c.target_diffusion_number) || c.target_diffusion_number <= 0.0 || c.target_diffusion_number > 0.5) { *msg = "adaptive target_diffusion_number must lie between 0 (exclusive) and 0.5"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!std::isfinite(c.max_growth_factor) || c.max_growth_factor < 1.0) { *msg = "adaptive max_growth_factor must be finite and at least 1"; return FLURSYS_ERR_INVALID_CONFIG; }
    }
    if (!(c.case_params.length > 0.0 && c.case_params.height > 0.0)) { *msg = "Domain dimensions must be positive"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (c.physics.energy_model != FLURSYS_ENERGY_OFF && c.physics.energy_model != FLURSYS_ENERGY_CONSTANT_PROPERTIES) { *msg = "unknown energy model"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    if (c.physics.buoyancy != FLURSYS_BUOYANCY_OFF && c.physics.buoyancy != FLURSYS_BUOYANCY_BOUSSINESQ) { *msg = "unknown buoyancy model"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    for (int s = 0; s < 4; ++s)
        if (c.physics.thermal[s].kind != FLURSYS_THERMAL_ADIABATIC && c.physics.thermal[s].kind != FLURSYS_THERMAL_FIXED_TEMPERATURE) { *msg = "unknown thermal boundary kind"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    // PhysicsSettings::validate at min_dt when adaptive, else dt (:180-189)
    const FlursysPhysicsSettings &ph = c.physics;
    const bool thermal = ph.energy_model == FLURSYS_ENERGY_CONSTANT_PROPERTIES;
    if (thermal) {
        if (!std::isfinite(ph.initial_temperature) || !std::isfinite(ph.thermal_diffusivity) || ph.thermal_diffusivity <= 0.0 || !std::isfinite(ph.source_temperature_rate)) { *msg = "thermal initial temperature, diffusivity, and source must be finite; diffusivity must be positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        for (int s = 0; s < 4; ++s)
            if (ph.thermal[s].kind == FLURSYS_THERMAL_FIXED_TEMPERATURE && !std::isfinite(ph.thermal[s].temperature)) { *msg = "fixed thermal boundary temperatures must be finite"; return FLURSYS_ERR_INVALID_CONFIG; }
        const double vdt = c.adaptive ? c.min_dt : c.dt;
        const double dx = c.case_params.length / c.nx, dy = c.case_params.height / c.ny;
        const double fourier = ph.thermal_diffusivity * vdt * (std::pow(1.0 / dx, 2) + std::pow(1.0 / dy, 2));
        if (fourier > 0.5) { *msg = "explicit thermal diffusion is unstable: alpha*dt*(1/dx^2 + 1/dy^2)=" + rust_sci(fourier, 3) + " exceeds 0.5"; return FLURSYS_ERR_INVALID_CONFIG; }
    }
    if (ph.buoyancy == FLURSYS_BUOYANCY_BOUSSINESQ) {
        if (!thermal) { *msg = "Boussinesq buoyancy requires the constant-property energy equation"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!std::isfinite(ph.reference_temperature) || !std::isfinite(ph.thermal_expansion) || ph.thermal_expansion < 0.0 || !std::isfinite(ph.gravity_x) || !std::isfinite(ph.gravity_y)) { *msg = "Boussinesq reference temperature, expansion coefficient, and gravity must be finite; expansion must be non-negative"; return FLURSYS_ERR_INVALID_CONFIG; }
    }
    return FLURSYS_OK;
}

}  // namespace

namespace flursys {

int32_t validate_config_checked(const FlursysCudaConfig &c, std::string *msg) { return validate_config(c, msg); }

void set_global_error(const std::string &msg) { g_error = msg; }

std::string rust_sci(double v, int prec) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.*e", prec, v);
    const std::string s(buf);
    const size_t e = s.find('e');
    if (e == std::string::npos) return s;
    return s.substr(0, e) + "e" + std::to_string(std::atoi(s.c_str() + e + 1));
}

std::string nonfinite_message(const char *name, unsigned long long index, const double *field, long long step,
                              bool two_d) {
    double v = NAN;
    if (field) cudaMemcpy(&v, field + index, sizeof v, cudaMemcpyDeviceToHost);
    const char *shown = std::isnan(v) ? "NaN" : (v > 0 ? "inf" : "-inf");
    char buf[256];
    if (two_d)
        std::snprintf(buf, sizeof buf, "Non-finite %s value at flat index %llu: %s (step %lld)", name, index, shown, step);
    else
        std::snprintf(buf, sizeof buf, "Non-finite 3D %s value at flat index %llu: %s", name, index, shown);
    return buf;
}

namespace {
std::atomic<int> g_injected_barrier_fault{0};
}

int take_injected_barrier_fault() { return g_injected_barrier_fault.exchange(0); }

int32_t set_cuda_error(std::string *dst, cudaError_t e, const char *what) {
    char buf[256];
    std::snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    *dst = buf;
    return e == cudaErrorMemoryAllocation ? FLURSYS_ERR_OUT_OF_MEMORY : FLURSYS_ERR_CUDA;
}

Pcg3dArgs make_pcg3d_args(PcgWorkspace &ws, int nx, int ny, int nz, double dx, double dy, double dz, double *x,
                          const double *rhs, int precision, int stop_rule, double tol, double atol, double rtol,
                          long long max_iters, int replace_every) {
    Pcg3dArgs a{};
    a.nx = nx; a.ny = ny; a.nz = nz;
    a.ix2 = 1.0 / (dx * dx); a.iy2 = 1.0 / (dy * dy); a.iz2 = 1.0 / (dz * dz);
    a.x = x; a.rhs = rhs;
    a.r = ws.r; a.d0 = ws.d0; a.d1 = ws.d1; a.q = ws.q; a.dx = ws.dx;
    a.partials = ws.partials; a.barrier = ws.barrier; a.result = ws.result;
    a.stop_rule = stop_rule; a.tol = tol; a.atol = atol; a.rtol = rtol;
    a.max_iters = max_iters; a.replace_every = replace_every > 0 ? replace_every : 50;
    a.precision_vec_width = precision == FLURSYS_PRECISION_MIXED ? 4 : 2;
    a.row_class = ws.row_class;
    return a;
}

// Enqueues one persistent 3D PCG solve of A x = -rhs on `stream`.
int32_t run_pcg3d(PcgWorkspace &ws, int nx, int ny, int nz, double dx, double dy, double dz, double *x,
                  const double *rhs, int precision, int stop_rule, double tol, double atol, double rtol,
                  long long max_iters, int replace_every, cudaStream_t stream, std::string *err) {
    Pcg3dArgs a = make_pcg3d_args(ws, nx, ny, nz, dx, dy, dz, x, rhs, precision, stop_rule, tol, atol, rtol, max_iters,
                                  replace_every);
    cudaError_t e = cudaMemsetAsync(ws.barrier, 0, sizeof(GridBarrier), stream);
    if (e == cudaSuccess) e = pcg3d_launch(a, ws.grid, precision, stream);
    if (e != cudaSuccess) return set_cuda_error(err, e, "pcg3d launch");
    return FLURSYS_OK;
}

cudaError_t PcgWorkspace::allocate(long long n, int precision, int device, int dim) {
    free_all();
    this->precision = precision;
    int maxgrid = 0;
    cudaError_t e = dim == 3 ? pcg3d_max_grid(precision, device, &maxgrid) : pcg2d_max_grid(precision, device, &maxgrid);
    if (e != cudaSuccess) return e;
    const int bs = dim == 3 ? pcg3d_block_size() : pcg2d_block_size();
    long long want = (n + (long long)bs * 4 - 1) / ((long long)bs * 4);  // >= 4 cells per thread
    grid = (int)std::max(1LL, std::min((long long)maxgrid, want));
    const size_t vb = precision == FLURSYS_PRECISION_MIXED ? sizeof(float) : sizeof(double);
    const int np = dim == 3 ? pcg3d_num_partials() : pcg2d_num_partials();
    if ((e = cudaMalloc(&r, vb * n)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&d0, vb * n)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&d1, vb * n)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&q, vb * n)) != cudaSuccess) return e;
    if (precision == FLURSYS_PRECISION_MIXED && (e = cudaMalloc(&dx, sizeof(float) * n)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&partials, sizeof(double) * (size_t)np * grid)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&barrier, sizeof(GridBarrier))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&result, sizeof(PcgResultDev))) != cudaSuccess) return e;
    if ((e = cudaMallocHost(&h_result, sizeof(PcgResultDev))) != cudaSuccess) return e;
    return cudaSuccess;
}

cudaError_t PcgWorkspace::allocate3d(int nx, int ny, int nz, int prec, int device, cudaStream_t stream) {
    cudaError_t e = allocate((long long)nx * ny * nz, prec, device, 3);
    if (e == cudaSuccess) e = pcg3d_make_row_class(ny, nz, &row_class, stream);
    return e;
}

void PcgWorkspace::free_all() {
    cudaFree(row_class);
    row_class = nullptr;
    cudaFree(r_z);
    r_z = nullptr;
    cudaFree(r); cudaFree(d0); cudaFree(d1); cudaFree(q); cudaFree(dx);
    cudaFree(partials); cudaFree(barrier); cudaFree(result);
    if (h_result) cudaFreeHost(h_result);
    r = d0 = d1 = q = nullptr; dx = nullptr; partials = nullptr; barrier = nullptr; result = nullptr;
    h_result = nullptr;
}

}  // namespace flursys

extern "C" {

uint32_t flursys_cuda_abi_version(void) { return FLURSYS_CUDA_ABI_VERSION; }

int32_t flursys_cuda_global_error(char *buf, size_t size) {
    copy_msg(g_error, buf, size);
    return FLURSYS_OK;
}

int32_t flursys_cuda_debug_inject_barrier_fault(int32_t extra_arrivals) {
    if (extra_arrivals < 0) {
        g_error = "extra_arrivals must be >= 0";
        return FLURSYS_ERR_INVALID_ARGUMENT;
    }
    g_injected_barrier_fault.store(extra_arrivals);
    return FLURSYS_OK;
}

// LidDrivenCavity3DConfig::default() (incompressible_3d.rs:27-47) for
// dimension 3; the CLI cavity defaults (src/bin/flursys.rs:102-123,236-300)
// with TimeStepSettings::default() (incompressible.rs:45-56) otherwise.
int32_t flursys_cuda_default_config(int32_t dimension, FlursysCudaConfig *c) {
    if (!c) { g_error = "null config"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    std::memset(c, 0, sizeof *c);
    c->abi_version = FLURSYS_CUDA_ABI_VERSION;
    c->dimension = dimension == 3 ? 3 : 2;
    c->case_params.kind = FLURSYS_CASE_CAVITY;
    c->case_params.length = 1.0;
    c->case_params.height = 1.0;
    // ThermalSettings::default (src/physics.rs:43-56); buoyancy off
    c->physics.initial_temperature = 293.15;
    c->physics.thermal_diffusivity = 2.2e-5;
    c->case_params.depth = 1.0;
    c->case_params.density = 1.0;
    c->case_params.reference_velocity = 1.0;
    c->case_params.reynolds = 100.0;
    c->case_params.kinematic_viscosity = 0.01;
    c->min_dt = 1.0e-6;
    c->max_dt = 1.0e-2;
    c->target_cfl = 0.5;
    c->target_diffusion_number = 0.25;
    c->max_growth_factor = 1.1;
    c->pressure_solver = FLURSYS_PRESSURE_PCG;
    c->pressure_atol = 0.0;
    c->pressure_rtol = 1.0e-8;
    c->precision = FLURSYS_PRECISION_F64;
    c->residual_replacement_every = 50;
    if (c->dimension == 3) {
        c->nx = c->ny = c->nz = 32;
        c->dt = 5.0e-4;
        c->max_steps = 10000;
        c->pressure_max_iters = 2000;
        c->pressure_tolerance = 1.0e-6;
        c->pressure_omega = 1.7;
        c->pressure_solver = FLURSYS_PRESSURE_SOR;
        c->stop_rule = FLURSYS_STOP_REFERENCE_RESIDUAL;
        c->convection = FLURSYS_CONVECTION_CENTRAL;
        c->t_end = 1e300;
    } else {
        c->nx = c->ny = 64;
        c->nz = 1;
        c->dt = 0.001;
        c->t_end = 100.0;
        c->max_steps = 100000;
        c->convection = FLURSYS_CONVECTION_UPWIND;
        c->coupling = FLURSYS_COUPLING_PROJECTION;
        c->stop_rule = FLURSYS_STOP_ABS_INF;
        c->pressure_max_iters = 1200;
        c->pressure_tolerance = 1.0e-5;
        c->pressure_omega = 1.7;
        c->velocity_relaxation = 0.7;
        c->pressure_relaxation = 0.3;
        c->steady_tolerance = 1.0e-7;
        c->minimum_steps = 2000;
    }
    return FLURSYS_OK;
}

int32_t flursys_cuda_create(const FlursysCudaConfig *cfg, FlursysCudaHandle **out) {
    if (!cfg || !out) { g_error = "null argument"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    *out = nullptr;
    std::string msg;
    int32_t st = validate_config(*cfg, &msg);
    if (st) { g_error = msg; return st; }
    auto *h = new FlursysCudaHandle();
    h->cfg = *cfg;
    st = handle_init(h, cfg);
    h->cfg.fcg_weights_path = nullptr;  // the path is read during create only
    if (st) {
        g_error = h->err;
        handle_free(h);
        delete h;
        return st;
    }
    *out = h;
    return FLURSYS_OK;
}

int32_t flursys_cuda_step(FlursysCudaHandle *h, int64_t nsteps, FlursysStepReport *report) {
    if (!h) { g_error = "null handle"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    if (nsteps < 0) { h->err = "nsteps must be non-negative"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return set_cuda_error(&h->err, e, "cudaSetDevice");
    FlursysStepReport rep;
    std::memset(&rep, 0, sizeof rep);
    int32_t st = FLURSYS_OK;
    for (int64_t s = 0; s < nsteps; ++s) {
        st = h->cfg.dimension == 3 ? step3d(h, &rep) : step2d(h, &rep);
        if (st) break;
        if (h->cfg.dimension == 2 && (rep.converged || rep.reached_end_time)) break;
    }
    if (report) *report = rep;
    return st;
}

size_t flursys_cuda_field_size(const FlursysCudaHandle *h, int32_t id) {
    if (!h) return 0;
    double *p = nullptr;
    size_t n = 0;
    field_ptr(const_cast<FlursysCudaHandle *>(h), id, &p, &n);
    return n;
}

int32_t flursys_cuda_download(FlursysCudaHandle *h, int32_t id, double *host, size_t n) {
    if (!h || !host) { g_error = "null argument"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    double *p = nullptr;
    size_t fn = 0;
    if (!field_ptr(h, id, &p, &fn)) { h->err = "unknown field id for this handle"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    if (fn != n) { h->err = "field size mismatch"; return FLURSYS_ERR_DIMENSION_MISMATCH; }
    cudaError_t e = cudaSetDevice(h->device);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, p, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return set_cuda_error(&h->err, e, "download");
    return FLURSYS_OK;
}

int32_t flursys_cuda_snapshot_begin(FlursysCudaHandle *h, const int32_t *ids, int32_t count, double *const *host,
                                    const size_t *sizes) {
    if (!h || (count > 0 && (!ids || !host || !sizes))) { g_error = "null argument"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    if (count < 0 || count > 16) { h->err = "a snapshot holds 1 to 16 fields"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    if (h->snap_pending) { h->err = "a snapshot is already pending on this handle"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    cudaError_t e = cudaSetDevice(h->device);
    if (e == cudaSuccess && !h->snap_stream) e = cudaStreamCreateWithFlags(&h->snap_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess && !h->snap_taken) e = cudaEventCreateWithFlags(&h->snap_taken, cudaEventDisableTiming);
    if (e == cudaSuccess && !h->snap_done) e = cudaEventCreateWithFlags(&h->snap_done, cudaEventDisableTiming);
    if (e != cudaSuccess) return set_cuda_error(&h->err, e, "snapshot set-up");
    for (int32_t i = 0; i < count; ++i) {
        double *p = nullptr;
        size_t fn = 0;
        if (!host[i] || !field_ptr(h, ids[i], &p, &fn)) { h->err = "unknown field id for this handle"; return FLURSYS_ERR_INVALID_ARGUMENT; }
        if (fn != sizes[i]) { h->err = "field size mismatch"; return FLURSYS_ERR_DIMENSION_MISMATCH; }
        if (h->snap_n[i] < fn) {
            cudaFree(h->snap_buf[i]);
            h->snap_buf[i] = nullptr;
            h->snap_n[i] = 0;
            e = cudaMalloc(&h->snap_buf[i], fn * sizeof(double));
            if (e != cudaSuccess) return set_cuda_error(&h->err, e, "snapshot buffer");
            h->snap_n[i] = fn;
        }
        e = cudaMemcpyAsync(h->snap_buf[i], p, fn * sizeof(double), cudaMemcpyDeviceToDevice, h->stream);
        if (e != cudaSuccess) return set_cuda_error(&h->err, e, "snapshot copy");
    }
    e = cudaEventRecord(h->snap_taken, h->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h->snap_stream, h->snap_taken, 0);
    for (int32_t i = 0; i < count && e == cudaSuccess; ++i)
        e = cudaMemcpyAsync(host[i], h->snap_buf[i], sizes[i] * sizeof(double), cudaMemcpyDeviceToHost, h->snap_stream);
    if (e == cudaSuccess) e = cudaEventRecord(h->snap_done, h->snap_stream);
    if (e != cudaSuccess) return set_cuda_error(&h->err, e, "snapshot drain");
    h->snap_pending = true;
    return FLURSYS_OK;
}

int32_t flursys_cuda_snapshot_wait(FlursysCudaHandle *h) {
    if (!h) { g_error = "null handle"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    if (!h->snap_pending) return FLURSYS_OK;
    h->snap_pending = false;
    const cudaError_t e = cudaEventSynchronize(h->snap_done);
    if (e != cudaSuccess) return set_cuda_error(&h->err, e, "snapshot wait");
    return FLURSYS_OK;
}

int32_t flursys_cuda_upload(FlursysCudaHandle *h, int32_t id, const double *host, size_t n) {
    if (!h || !host) { g_error = "null argument"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    double *p = nullptr;
    size_t fn = 0;
    if (!field_ptr(h, id, &p, &fn)) { h->err = "unknown field id for this handle"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    if (fn != n) { h->err = "field size mismatch"; return FLURSYS_ERR_DIMENSION_MISMATCH; }
    cudaError_t e = cudaSetDevice(h->device);
    if (e == cudaSuccess) e = cudaMemcpyAsync(p, host, n * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return set_cuda_error(&h->err, e, "upload");
    if (h->cfg.dimension == 2) on_upload2d(h, id);
    return FLURSYS_OK;
}

int32_t flursys_cuda_state(const FlursysCudaHandle *h, int64_t *step, double *time) {
    if (!h) { g_error = "null handle"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    if (step) *step = h->step;
    if (time) *time = h->time;
    return FLURSYS_OK;
}

int32_t flursys_cuda_set_stream(FlursysCudaHandle *h, void *stream) {
    if (!h) { g_error = "null handle"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    h->stream = stream ? static_cast<cudaStream_t>(stream) : h->own_stream;
    return FLURSYS_OK;
}

int32_t flursys_cuda_solver_profile(const FlursysCudaHandle *h, double *phase_ms, size_t n) {
    if (!h || !phase_ms) { g_error = "null argument"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    const PcgResultDev *r = h->pcg.h_result;
    for (size_t i = 0; i < n && i < 6; ++i) phase_ms[i] = r ? 1e-6 * (double)r->phase_ns[i] : 0.0;
    return FLURSYS_OK;
}

int32_t flursys_cuda_solve_kind(const FlursysCudaHandle *h, int32_t *kind) {
    if (!h || !kind) { g_error = "null argument"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    if (h->cfg.dimension != 3) { g_error = "the solve kind describes 3D handles"; return FLURSYS_ERR_INVALID_ARGUMENT; }
    if (h->cfg.pressure_solver == FLURSYS_PRESSURE_FCG) *kind = FLURSYS_SOLVE_FCG;
    else if (h->cfg.pressure_solver == FLURSYS_PRESSURE_SOR) *kind = FLURSYS_SOLVE_SOR;
    else if (!h->use_seq) *kind = FLURSYS_SOLVE_PERSISTENT;
    else if (h->seq.resident) *kind = FLURSYS_SOLVE_RESIDENT;
    else *kind = FLURSYS_SOLVE_GRAPH;
    return FLURSYS_OK;
}

int32_t flursys_cuda_last_error(const FlursysCudaHandle *h, char *buf, size_t size) {
    copy_msg(h ? h->err : g_error, buf, size);
    return FLURSYS_OK;
}

int32_t flursys_cuda_destroy(FlursysCudaHandle *h) {
    if (!h) return FLURSYS_OK;
    cudaSetDevice(h->device);
    if (h->snap_pending) cudaEventSynchronize(h->snap_done);
    for (double *b : h->snap_buf) cudaFree(b);
    if (h->snap_taken) cudaEventDestroy(h->snap_taken);
    if (h->snap_done) cudaEventDestroy(h->snap_done);
    if (h->snap_stream) cudaStreamDestroy(h->snap_stream);
    handle_free(h);
    delete h;
    return FLURSYS_OK;
}

}  // extern "C"
