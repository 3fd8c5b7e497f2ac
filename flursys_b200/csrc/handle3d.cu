// handle3d.cu — LidDrivenCavity3DSolver on the device: allocation, one
// advance_one_step (src/solver/incompressible_3d.rs:164-172) and field access.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "capi_internal.cuh"
#include "sor.cuh"

namespace flursys {

int32_t pcg_result_status(const PcgResultDev &r, std::string *err) {
    if (r.device_error & kDevErrBarrierTimeout) {
        *err = "pressure solver: a device grid barrier timed out";
        return FLURSYS_ERR_TIMEOUT;
    }
    if (r.error == FLURSYS_ERR_BREAKDOWN) {
        *err = "PCG pressure solver encountered a singular search direction";
        return FLURSYS_ERR_BREAKDOWN;
    }
    if (r.error == FLURSYS_ERR_NON_FINITE) {
        *err = "PCG pressure solver produced a non-finite residual";
        return FLURSYS_ERR_NON_FINITE;
    }
    if (r.error != 0) {
        *err = "pressure solver failed";
        return r.error;
    }
    return FLURSYS_OK;
}

static int32_t init3d(FlursysCudaHandle *h) {
    const FlursysCudaConfig &c = h->cfg;
    Cavity3dState &s = h->s3;
    s.nx = (int)c.nx; s.ny = (int)c.ny; s.nz = (int)c.nz; s.sms = h->sms;
    s.dx = c.case_params.length / c.nx;
    s.dy = c.case_params.height / c.ny;
    s.dz = c.case_params.depth / c.nz;
    s.lid = c.case_params.reference_velocity;
    s.rho = c.case_params.density;
    s.nu = s.lid * c.case_params.length / c.case_params.reynolds;  // viscosity() :86-88
    const long long nc = c.nx * c.ny * c.nz;
    const long long nu = (c.nx + 1) * c.ny * c.nz, nv = c.nx * (c.ny + 1) * c.nz, nw = c.nx * c.ny * (c.nz + 1);
    double **bufs[8] = {&s.u, &s.v, &s.w, &s.us, &s.vs, &s.ws, &s.p, &s.rhs};
    long long sizes[8] = {nu, nv, nw, nu, nv, nw, nc, nc};
    for (int b = 0; b < 8; ++b) {
        cudaError_t e = cudaMalloc(bufs[b], sizeof(double) * sizes[b]);
        if (e == cudaSuccess) e = cudaMemsetAsync(*bufs[b], 0, sizeof(double) * sizes[b], h->stream);
        if (e != cudaSuccess) return set_cuda_error(&h->err, e, "allocating 3D fields");
    }
    cudaError_t e = cudaMalloc(&h->diag3, sizeof(Diag3Dev));
    if (e == cudaSuccess) e = cudaMallocHost(&h->h_diag3, sizeof(Diag3Dev));
    if (e == cudaSuccess) e = h->pcg.allocate3d((int)c.nx, (int)c.ny, (int)c.nz, c.precision, h->device, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return set_cuda_error(&h->err, e, "allocating 3D solver workspace");
    if (c.pressure_solver == FLURSYS_PRESSURE_FCG) {
        if (!c.fcg_weights_path || !c.fcg_weights_path[0]) {
            h->err = "pressure_solver fcg needs fcg_weights_path (a trained network)";
            return FLURSYS_ERR_INVALID_CONFIG;
        }
        if (c.nx % 8 || c.ny % 8 || c.nz % 8) {
            h->err = "the learned FCG needs nx, ny and nz divisible by 8";
            return FLURSYS_ERR_UNSUPPORTED;
        }
        std::vector<float> params;
        int32_t st = fcgnet_read_file(c.fcg_weights_path, &params, &h->err);
        if (!st) st = fcgnet_create(params.data(), &h->fcg_net, &h->err);
        if (st) return st;
        return FLURSYS_OK;
    }
    // The graph-driven PCG is the default; FLURSYS_PCG_VARIANT=persistent
    // selects the single cooperative kernel instead.
    const char *variant = std::getenv("FLURSYS_PCG_VARIANT");
    h->use_seq = c.pressure_solver != FLURSYS_PRESSURE_SOR && !(variant && std::strcmp(variant, "persistent") == 0);
    if (h->use_seq) {
        const int rule = c.stop_rule == FLURSYS_STOP_REFERENCE_RESIDUAL ? FLURSYS_STOP_ABS_INF : c.stop_rule;
        Pcg3dArgs a = make_pcg3d_args(h->pcg, s.nx, s.ny, s.nz, s.dx, s.dy, s.dz, s.p, s.rhs, c.precision, rule,
                                      c.pressure_tolerance, c.pressure_atol, c.pressure_rtol, c.pressure_max_iters,
                                      c.residual_replacement_every);
        e = pcg3d_seq_plan(h->seq, a, c.precision, h->device);
        if (e == cudaSuccess) e = cudaMallocHost(&h->h_seq, sizeof(CgSeqState));
        if (e != cudaSuccess) return set_cuda_error(&h->err, e, "building the pressure-solve graph");
    }
    return FLURSYS_OK;
}

int32_t handle_init(FlursysCudaHandle *h, const FlursysCudaConfig *cfg) {
    h->device = cfg->device;
    cudaError_t e = cudaSetDevice(h->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking);
    for (int i = 0; i < 4 && e == cudaSuccess; ++i) e = cudaEventCreate(&h->ev[i]);
    if (e != cudaSuccess) return set_cuda_error(&h->err, e, "CUDA initialisation");
    h->stream = h->own_stream;
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, h->device);
    if (!coop) {
        h->err = "device does not support cooperative launches";
        return FLURSYS_ERR_UNSUPPORTED;
    }
    if (cfg->dimension == 3) return init3d(h);
    return init2d(h);
}

void handle_free(FlursysCudaHandle *h) {
    if (h->cfg.dimension == 2) free2d(h);
    Cavity3dState &s = h->s3;
    double *bufs[8] = {s.u, s.v, s.w, s.us, s.vs, s.ws, s.p, s.rhs};
    for (double *b : bufs) cudaFree(b);
    cudaFree(h->diag3);
    if (h->h_diag3) cudaFreeHost(h->h_diag3);
    h->pcg.free_all();
    pcg3d_seq_destroy(h->seq);
    if (h->fcg_net) fcgnet_destroy(h->fcg_net);
    h->fcg_net = nullptr;
    if (h->h_seq) cudaFreeHost(h->h_seq);
    for (auto &ev : h->ev)
        if (ev) cudaEventDestroy(ev);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
}

int32_t step3d(FlursysCudaHandle *h, FlursysStepReport *rep) {
    const FlursysCudaConfig &c = h->cfg;
    Cavity3dState &s = h->s3;
    const double dt = c.dt;
    cudaStream_t st = h->stream;
    cudaError_t e = cudaEventRecord(h->ev[0], st);
    if (e == cudaSuccess) e = cavity3d_predict(s, dt, st);
    if (e == cudaSuccess) e = cavity3d_rhs(s, dt, st);
    if (e == cudaSuccess) e = cudaEventRecord(h->ev[1], st);
    if (e != cudaSuccess) return set_cuda_error(&h->err, e, "3D predictor");
    int32_t status;
    const bool sor = c.pressure_solver == FLURSYS_PRESSURE_SOR;
    const bool fcg = c.pressure_solver == FLURSYS_PRESSURE_FCG;
    if (fcg) {
        status = fcg_solve(h->fcg_net, s.nx, s.ny, s.nz, s.dx, s.dy, s.dz, s.p, s.rhs, c.pressure_atol,
                           c.pressure_rtol, c.pressure_max_iters, c.precision, st, &h->fcg_report, &h->err);
        if (!status) {
            const FlursysFcgReport &f = h->fcg_report;
            PcgResultDev &m = *h->pcg.h_result;
            std::memset(&m, 0, sizeof m);
            m.status = f.status;
            m.iterations = f.fcg_iterations + f.pcg_iterations;
            m.initial = f.initial_residual;
            m.residual = f.final_residual;
            m.true_l2 = f.final_residual;
            m.initial_l2 = f.initial_residual;
        }
    } else if (sor) {
        status = run_sor3d(h->pcg, s.nx, s.ny, s.nz, s.dx, s.dy, s.dz, s.p, s.rhs, c.pressure_omega,
                           c.pressure_tolerance, c.pressure_max_iters, st, &h->err);
    } else if (h->use_seq) {
        const cudaError_t le = pcg3d_seq_launch(h->seq, st);
        status = le == cudaSuccess ? FLURSYS_OK : set_cuda_error(&h->err, le, "pressure-solve graph");
    } else {
        const int rule = c.stop_rule == FLURSYS_STOP_REFERENCE_RESIDUAL ? FLURSYS_STOP_ABS_INF : c.stop_rule;
        status = run_pcg3d(h->pcg, s.nx, s.ny, s.nz, s.dx, s.dy, s.dz, s.p, s.rhs, c.precision, rule,
                           c.pressure_tolerance, c.pressure_atol, c.pressure_rtol, c.pressure_max_iters,
                           c.residual_replacement_every, st, &h->err);
    }
    if (status) return status;
    e = cudaEventRecord(h->ev[2], st);
    if (e == cudaSuccess) e = cavity3d_correct(s, dt, st);
    if (e == cudaSuccess) e = cavity3d_diagnostics(s, h->diag3, st);
    if (e == cudaSuccess) e = cudaEventRecord(h->ev[3], st);
    if (e == cudaSuccess) {
        if (h->use_seq && !sor && !fcg)
            e = cudaMemcpyAsync(h->h_seq, h->seq.state, sizeof(CgSeqState), cudaMemcpyDeviceToHost, st);
        else if (!fcg)
            e = cudaMemcpyAsync(h->pcg.h_result, h->pcg.result, sizeof(PcgResultDev), cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->h_diag3, h->diag3, sizeof(Diag3Dev), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return set_cuda_error(&h->err, e, "3D step");
    if (h->use_seq && !sor && !fcg) {
        const CgSeqState &q = *h->h_seq;
        PcgResultDev &m = *h->pcg.h_result;  // the shared result record
        m.error = q.error;
        m.status = q.status;
        m.iterations = q.iterations;
        m.initial = q.initial;
        m.residual = q.residual;
        m.true_l2 = q.true_l2;
        m.initial_l2 = q.initial_l2;
        m.device_error = q.device_error;
        for (int i = 0; i < 6; ++i) m.phase_ns[i] = q.phase_ns[i];
    }
    const PcgResultDev &r = *h->pcg.h_result;
    status = pcg_result_status(r, &h->err);
    if (status) return status;
    h->step += 1;
    h->time = h->step * dt;
    // ensure_finite (incompressible_3d.rs:534-554)
    const char *names[4] = {"pressure", "u", "v", "w"};
    const double *fields[4] = {h->s3.p, h->s3.u, h->s3.v, h->s3.w};
    for (int f = 0; f < 4; ++f) {
        if (h->h_diag3->bad_index[f] != ~0ull) {
            h->err = nonfinite_message(names[f], h->h_diag3->bad_index[f], fields[f], h->step, false);
            return FLURSYS_ERR_NON_FINITE;
        }
    }
    float ms_step = 0.f, ms_p = 0.f;
    cudaEventElapsedTime(&ms_step, h->ev[0], h->ev[3]);
    cudaEventElapsedTime(&ms_p, h->ev[1], h->ev[2]);
    std::memset(rep, 0, sizeof *rep);
    rep->iteration = h->step;
    rep->time = h->time;
    rep->time_step = dt;
    rep->continuity_residual = h->h_diag3->max_divergence;
    rep->pressure_residual = r.residual;
    rep->pressure_iterations = r.iterations;
    rep->max_speed = h->h_diag3->max_speed;
    rep->pressure_initial_residual = r.initial;
    rep->pressure_true_relative_residual = r.initial_l2 > 0.0 ? r.true_l2 / r.initial_l2 : 0.0;
    rep->pressure_solve_ms = ms_p;
    rep->step_ms = ms_step;
    rep->pressure_status = r.status;
    rep->fcg_fallback = fcg ? h->fcg_report.fallback : 0;
    return FLURSYS_OK;
}

bool field_ptr(FlursysCudaHandle *h, int32_t id, double **p, size_t *n) {
    if (h->cfg.dimension == 2) return field_ptr2d(h, id, p, n);
    const FlursysCudaConfig &c = h->cfg;
    const Cavity3dState &s = h->s3;
    const size_t nc = c.nx * c.ny * c.nz;
    const size_t nu = (c.nx + 1) * c.ny * c.nz, nv = c.nx * (c.ny + 1) * c.nz, nw = c.nx * c.ny * (c.nz + 1);
    switch (id) {
        case FLURSYS_FIELD_U: *p = s.u; *n = nu; return true;
        case FLURSYS_FIELD_V: *p = s.v; *n = nv; return true;
        case FLURSYS_FIELD_W: *p = s.w; *n = nw; return true;
        case FLURSYS_FIELD_PRESSURE: *p = s.p; *n = nc; return true;
        case FLURSYS_FIELD_RHS: *p = s.rhs; *n = nc; return true;
        case FLURSYS_FIELD_U_STAR: *p = s.us; *n = nu; return true;
        case FLURSYS_FIELD_V_STAR: *p = s.vs; *n = nv; return true;
        case FLURSYS_FIELD_W_STAR: *p = s.ws; *n = nw; return true;
        default: *p = nullptr; *n = 0; return false;
    }
}

}  // namespace flursys

extern "C" int32_t flursys_cuda_stencil_pcg(int64_t nx, int64_t ny, int64_t nz, double dx, double dy, double dz,
                                            const double *rhs, double *x_inout, int32_t precision,
                                            const FlursysLinearSolverOptions *options,
                                            FlursysLinearSolveReport *report) {
    using namespace flursys;
    if (!rhs || !x_inout || !options || nx < 1 || ny < 1 || nz < 1) return FLURSYS_ERR_INVALID_ARGUMENT;
    if (precision != FLURSYS_PRECISION_F64 && precision != FLURSYS_PRECISION_MIXED) return FLURSYS_ERR_INVALID_ARGUMENT;
    if (!(std::isfinite(options->absolute_tolerance) && options->absolute_tolerance >= 0.0 &&
          std::isfinite(options->relative_tolerance) && options->relative_tolerance >= 0.0))
        return FLURSYS_ERR_BREAKDOWN;  // validate_solve_inputs (src/linear/solver.rs:282-291)
    if (nz == 1) return stencil_pcg2d(nx, ny, dx, dy, rhs, x_inout, precision, options, report);
    const long long n = nx * ny * nz;
    int device = 0;
    cudaGetDevice(&device);
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return FLURSYS_ERR_CUDA;
    PcgWorkspace ws;
    double *dxp = nullptr, *drhs = nullptr;
    std::string err;
    int32_t status = FLURSYS_OK;
    if (n >= (1LL << 31)) return FLURSYS_ERR_INVALID_ARGUMENT;
    cudaError_t e = ws.allocate3d((int)nx, (int)ny, (int)nz, precision, device, st);
    if (e == cudaSuccess) e = cudaMalloc(&dxp, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&drhs, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dxp, x_inout, sizeof(double) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(drhs, rhs, sizeof(double) * n, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) status = set_cuda_error(&err, e, "stencil PCG setup");
    if (!status)
        status = run_pcg3d(ws, (int)nx, (int)ny, (int)nz, dx, dy, dz, dxp, drhs, precision, FLURSYS_STOP_REL_L2, 0.0,
                           options->absolute_tolerance, options->relative_tolerance, options->max_iterations, 50, st,
                           &err);
    if (!status) {
        e = cudaMemcpyAsync(ws.h_result, ws.result, sizeof(PcgResultDev), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(x_inout, dxp, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) status = set_cuda_error(&err, e, "stencil PCG");
    }
    if (!status) status = pcg_result_status(*ws.h_result, &err);
    if (!status && report) {
        const PcgResultDev &r = *ws.h_result;
        report->status = r.status;
        report->reserved = 0;
        report->iterations = r.iterations;
        report->initial_residual = r.initial;
        report->final_residual = r.residual;
        report->relative_residual = r.initial == 0.0 ? 0.0 : r.residual / r.initial;
    }
    ws.free_all();
    cudaFree(dxp);
    cudaFree(drhs);
    cudaStreamDestroy(st);
    if (status) set_global_error(err);
    return status;
}

