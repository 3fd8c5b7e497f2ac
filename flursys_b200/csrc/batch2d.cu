// batch2d.cu — many independent 2D projection solvers of uneven size
// advanced together on one device (flursys_cuda_batch_*).
//
// Each instance is one IncompressibleSolver (src/solver/incompressible.rs)
// with its own grid, viscosity, dt control and t_end. Its state lives in one
// pooled device allocation and its controls (dt, time, step, max |u|, max |v|,
// active flag, status) in a device-resident BatchCtl record, so a whole step
// runs without the host:
//
//   batch_begin        one block: per instance the dt rule of advance_one_step
//                      (:622-650, adaptive_time_step :2308-2336, the t_end
//                      clamp), reset of its barrier and non-finite indices;
//                      then the pressure blocks are shared out in proportion
//                      to cells x pressure iterations of the previous step
//   predict, bnd, rhs  persistent kernels over a table of tiles
//                      (instance, first element); tiles of stopped instances
//                      are skipped
//   pcg2d              one cooperative launch, each instance on its own block
//                      range with its own bounded barrier (pcg2d.cu)
//   correct, bnd, post persistent tile kernels as above; post leaves one
//                      partial record per tile
//   batch_end          one block per instance: fixed-order reduction of its
//                      tiles, error checks, u/un and v/vn pointer swap in the
//                      control record, time/step update and the report
//
// One step is captured once as a CUDA graph and replayed; the pointer swap in
// device memory makes every replay identical. The element work is shared with
// the single-grid kernels (cavity2d_dev.cuh), so an instance computes what a
// single-grid handle with the same config computes.
//
// The autotuner (FLURSYS_BATCH_AUTOTUNE) times each tile kernel at several
// tile sizes on the initial state (all of them are idempotent there) and the
// pressure kernel at several blocks per SM on a synthetic right-hand side
// (restored to zero afterwards), and keeps the fastest of each.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "capi_internal.cuh"
#include "cavity2d.cuh"
#include "cavity2d_dev.cuh"
#include "common.cuh"
#include "flursys_cuda.h"
#include "pcg2d.cuh"

namespace flursys {

namespace {

constexpr int kBlk = 256;
constexpr int kPostParts = 8;

enum BatchOp { kOpPredict = 0, kOpBndStar = 1, kOpRhs = 2, kOpCorrect = 3, kOpBndNew = 4, kOpPost = 5, kNumOps = 6 };

// Device-resident controls of one instance.
struct BatchCtl {
    Cavity2dState s;
    // SimulationConfig time control (incompressible.rs:93-191)
    double dt_cfg, min_dt, max_dt, target_cfl, target_diff, max_growth, t_end;
    double steady_tol, pressure_tol, force_q;
    long long minimum_steps;
    int adaptive, case_kind;
    // evolving state
    double current_dt, time, step_dt, max_u, max_v;
    long long step, last_iters;
    int active;   // 1 while the instance steps
    int status;   // FlursysStatus: OK, REACHED_END_TIME or the error that stopped it
    int post_t0, post_t1;  // its tiles in the post table
    long long cells;
};

__device__ __forceinline__ bool reached_end(const BatchCtl &c) {
    const double tol = 2.220446049250313e-16 * fmax(fabs(c.t_end), 1.0) * 16.0;
    return c.time >= c.t_end - tol;
}

// Elements of one instance that an op covers.
__host__ __device__ __forceinline__ int op_elems(int op, int nx, int ny) {
    const int nc = nx * ny, nu = (nx + 1) * ny, nv = nx * (ny + 1);
    switch (op) {
        case kOpPredict:
        case kOpCorrect: return nu + nv;
        case kOpBndStar:
        case kOpBndNew: return nx > ny ? nx : ny;
        case kOpRhs: return nc;
        default: return nu > nv ? (nu > nc ? nu : nc) : (nv > nc ? nv : nc);
    }
}

// Pressure blocks in proportion to cells x iterations of the previous step
// (an estimate of 4 sqrt(cells) before the first one); one block at least,
// and no more than one per kBlk cells. Run by one thread.
__device__ void share_pressure_blocks(const BatchCtl *ctl, Pcg2dInstance *pin, int n, int total_blocks) {
    double wsum = 0.0;
    int nact = 0;
    for (int t = 0; t < n; ++t) {
        if (!ctl[t].active) continue;
        const double cells = double(ctl[t].cells);
        const double its = ctl[t].last_iters > 0 ? double(ctl[t].last_iters) : 4.0 * sqrt(cells);
        wsum += cells * its;
        ++nact;
    }
    const int avail = total_blocks - nact;
    int b0 = 0;
    for (int t = 0; t < n; ++t) {
        pin[t].block0 = b0;
        if (!ctl[t].active) {
            pin[t].nblocks = 0;
            continue;
        }
        const double cells = double(ctl[t].cells);
        const double its = ctl[t].last_iters > 0 ? double(ctl[t].last_iters) : 4.0 * sqrt(cells);
        long long nb = 1 + (avail > 0 && wsum > 0.0 ? (long long)floor(double(avail) * (cells * its) / wsum) : 0);
        const long long cap = (ctl[t].cells + kBlk - 1) / kBlk;
        if (nb > cap) nb = cap;
        pin[t].nblocks = (int)nb;
        b0 += (int)nb;
    }
}

__device__ __forceinline__ void reset_barrier(GridBarrier *b) {
    b->count = 0u;
    b->generation = 0u;
    b->error = 0u;
}

// Pressure launch set-up alone (tuning runs): barriers and block shares.
__global__ void batch_prepare_pressure(const BatchCtl *ctl, Pcg2dInstance *pin, int n, int total_blocks) {
    for (int t = threadIdx.x; t < n; t += blockDim.x) reset_barrier(pin[t].barrier);
    __syncthreads();
    if (threadIdx.x == 0) share_pressure_blocks(ctl, pin, n, total_blocks);
}

__global__ void batch_begin(BatchCtl *ctl, Pcg2dInstance *pin, int n, int total_blocks) {
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        BatchCtl &c = ctl[t];
        for (int f = 0; f < 4; ++f) c.s.diag->bad_index[f] = ~0ull;
        reset_barrier(pin[t].barrier);
        if (!c.active) continue;
        if (reached_end(c)) {
            c.active = 0;
            c.status = FLURSYS_ERR_REACHED_END_TIME;
            continue;
        }
        double dt = c.dt_cfg;
        if (c.adaptive) {
            // adaptive_time_step (:2308-2336), the same expression as the host rule
            const double rate = c.max_u / c.s.dx + c.max_v / c.s.dy;
            const double cfl_dt = rate > 2.220446049250313e-16 ? c.target_cfl / rate : c.max_dt;
            const double inv = 1.0 / (c.s.dx * c.s.dx) + 1.0 / (c.s.dy * c.s.dy);
            const double diff_dt = c.target_diff / (c.s.nu * inv);
            const double stable = fmin(fmin(c.max_dt, cfl_dt), diff_dt);
            if (stable < c.min_dt) {
                c.active = 0;
                c.status = FLURSYS_ERR_INVALID_CONFIG;
                continue;
            }
            dt = fmin(fmax(fmin(stable, c.current_dt * c.max_growth), c.min_dt), c.max_dt);
        }
        dt = fmin(dt, c.t_end - c.time);
        if (dt <= 0.0) {
            c.active = 0;
            c.status = FLURSYS_ERR_REACHED_END_TIME;
            continue;
        }
        if (c.adaptive) c.current_dt = dt;
        c.step_dt = dt;
    }
    __syncthreads();
    if (threadIdx.x == 0) share_pressure_blocks(ctl, pin, n, total_blocks);
}

template <int OP>
__global__ void __launch_bounds__(kBlk) batch_tiles(const BatchCtl *__restrict__ ctl, const int2 *__restrict__ tiles,
                                                    int ntiles, int tile_elems, double *__restrict__ post_partials) {
    __shared__ double red[kBlk / 32];
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int2 tl = tiles[t];
        const BatchCtl *c = ctl + tl.x;
        if (!c->active) continue;  // uniform over the block
        const Cavity2dState s = c->s;
        const double dt = c->step_dt;
        const int end = min(tl.y + tile_elems, op_elems(OP, s.nx, s.ny));
        if (OP == kOpPost) {
            PostAcc a;
            for (int id = tl.y + threadIdx.x; id < end; id += kBlk) post_elem(s, id, a);
            const double vals[kPostParts] = {a.mdiv, a.mspeed, a.mu, a.mv, a.du, a.dv, a.fx, a.fy};
            for (int k = 0; k < kPostParts; ++k) {
                const double v = k < 6 ? block_max<kBlk>(vals[k], red) : block_sum<kBlk>(vals[k], red);
                if (threadIdx.x == 0) post_partials[(long long)t * kPostParts + k] = v;
            }
            continue;
        }
        for (int id = tl.y + threadIdx.x; id < end; id += kBlk) {
            if (OP == kOpPredict) predict_elem(s, id, dt, 0, 1.0);
            else if (OP == kOpBndStar) boundary_elem(s, s.us, s.vs, id);
            else if (OP == kOpRhs) rhs_elem(s, id, s.rho / dt);
            else if (OP == kOpCorrect) correct_elem(s, id, dt / s.rho);
            else boundary_elem(s, s.un, s.vn, id);
        }
    }
}

__global__ void __launch_bounds__(kBlk) batch_end(BatchCtl *ctl, const PcgResultDev *res, const double *post_partials,
                                                  FlursysStepReport *rep, unsigned *dev_err) {
    __shared__ double red[kBlk / 32];
    BatchCtl &c = ctl[blockIdx.x];
    if (!c.active) return;  // uniform over the block
    double out[kPostParts];
    for (int k = 0; k < kPostParts; ++k) {
        double a = 0.0;
        for (int t = c.post_t0 + threadIdx.x; t < c.post_t1; t += kBlk) {
            const double v = post_partials[(long long)t * kPostParts + k];
            a = k < 6 ? fmax(a, v) : a + v;
        }
        out[k] = k < 6 ? block_max<kBlk>(a, red) : block_sum<kBlk>(a, red);
    }
    if (threadIdx.x != 0) return;
    const PcgResultDev &r = res[blockIdx.x];
    if (r.device_error) {
        atomicOr(dev_err, r.device_error);
        c.active = 0;
        c.status = FLURSYS_ERR_TIMEOUT;
        return;
    }
    int err = r.error;
    const Diag2Dev &d = *c.s.diag;
    for (int f = 0; f < 4 && !err; ++f)
        if (d.bad_index[f] != ~0ull) err = FLURSYS_ERR_NON_FINITE;
    if (err) {  // the step is not taken, as when advance_one_step returns Err
        c.active = 0;
        c.status = err;
        return;
    }
    double *t0 = c.s.u; c.s.u = c.s.un; c.s.un = t0;
    double *t1 = c.s.v; c.s.v = c.s.vn; c.s.vn = t1;
    c.step += 1;
    c.time += c.step_dt;
    c.max_u = out[2];
    c.max_v = out[3];
    c.last_iters = r.iterations;
    FlursysStepReport &o = rep[blockIdx.x];
    const double dx = c.s.dx, dy = c.s.dy;
    o.iteration = c.step;
    o.time = c.time;
    o.time_step = c.step_dt;
    o.continuity_residual = out[0];
    o.pressure_residual = r.residual;
    o.pressure_iterations = r.iterations;
    o.momentum_residual = fmax(out[4], out[5]);
    o.max_speed = out[1];
    o.momentum_cfl = c.step_dt * (out[2] / dx + out[3] / dy);
    o.viscous_diffusion_number = c.s.nu * c.step_dt * (1.0 / (dx * dx) + 1.0 / (dy * dy));
    o.drag_coefficient = c.s.cylinder && c.force_q > 0.0 ? out[6] / c.force_q : 0.0;
    o.lift_coefficient = c.s.cylinder && c.force_q > 0.0 ? out[7] / c.force_q : 0.0;
    o.converged = c.case_kind != FLURSYS_CASE_CYLINDER && c.step >= c.minimum_steps &&
                  o.momentum_residual < c.steady_tol && o.continuity_residual < 10.0 * c.pressure_tol;
    o.reached_end_time = reached_end(c) ? 1 : 0;
    o.pressure_initial_residual = r.initial;
    o.pressure_true_relative_residual = r.initial_l2 > 0.0 ? r.true_l2 / r.initial_l2 : 0.0;
    o.pressure_solve_ms = 0.0;
    o.step_ms = 0.0;
    o.pressure_status = r.status;
    o.fcg_fallback = 0;
}

// Seeded synthetic right-hand side of the pressure tuning runs (fluid cells).
__global__ void synth_rhs(double *rhs, const uint8_t *flags, int n, unsigned seed) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        unsigned h = (unsigned)c * 2654435761u ^ seed;
        h ^= h >> 16; h *= 2246822519u; h ^= h >> 13; h *= 3266489917u; h ^= h >> 16;
        rhs[c] = (flags[c] & 3) ? 0.0 : (double(h) * (1.0 / 4294967296.0) - 0.5);
    }
}

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

}  // namespace flursys

using namespace flursys;

struct FlursysBatchHandle {
    int n = 0;
    int precision = 0;
    int device = 0, sms = 0;
    cudaStream_t stream = nullptr;
    char *pool = nullptr;
    size_t pool_bytes = 0;
    BatchCtl *ctl = nullptr;             // device
    std::vector<BatchCtl> h_ctl;         // host copy (layout + pointers)
    Pcg2dInstance *pin = nullptr;        // device
    std::vector<Pcg2dInstance> h_pin;
    PcgResultDev *res = nullptr;         // device, one per instance
    FlursysStepReport *rep = nullptr;    // device, one per instance
    FlursysStepReport *h_rep = nullptr;  // pinned
    BatchCtl *h_ctl_pinned = nullptr;    // pinned copy for reports
    unsigned *dev_err = nullptr;
    unsigned *h_dev_err = nullptr;
    double *post_partials = nullptr;
    int2 *tiles[kNumOps] = {};
    int ntiles[kNumOps] = {};
    int tile_elems[kNumOps] = {};
    int grid[kNumOps] = {};
    int pcg_blocks = 0, pcg_per_sm = 0, pcg_max_per_sm = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graph_nodes = 0;
    bool use_graph = true;
    double tune_ms = 0.0;
    double last_step_ms = 0.0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<int> nx, ny;
};

namespace {

int32_t fail(const std::string &msg, int32_t code) {
    set_global_error(msg);
    return code;
}

int32_t cuda_fail(cudaError_t e, const char *what) {
    std::string m;
    const int32_t code = set_cuda_error(&m, e, what);
    set_global_error(m);
    return code;
}

// Tile table of one op at `elems` elements per tile; returns the post tile
// ranges per instance when op == kOpPost.
std::vector<int2> make_tiles(const FlursysBatchHandle *h, int op, int elems, std::vector<int> *first) {
    std::vector<int2> t;
    if (first) first->assign(h->n + 1, 0);
    for (int i = 0; i < h->n; ++i) {
        if (first) (*first)[i] = (int)t.size();
        const int m = op_elems(op, h->nx[i], h->ny[i]);
        for (int s = 0; s < m; s += elems) t.push_back(make_int2(i, s));
    }
    if (first) (*first)[h->n] = (int)t.size();
    return t;
}

template <int OP>
int occupancy_blocks(int sms) {
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, batch_tiles<OP>, kBlk, 0);
    return sms * std::max(per, 1);
}

int max_grid(int op, int sms) {
    switch (op) {
        case kOpPredict: return occupancy_blocks<kOpPredict>(sms);
        case kOpBndStar: return occupancy_blocks<kOpBndStar>(sms);
        case kOpRhs: return occupancy_blocks<kOpRhs>(sms);
        case kOpCorrect: return occupancy_blocks<kOpCorrect>(sms);
        case kOpBndNew: return occupancy_blocks<kOpBndNew>(sms);
        default: return occupancy_blocks<kOpPost>(sms);
    }
}

cudaError_t launch_op(FlursysBatchHandle *h, int op, cudaStream_t st) {
    const int g = h->grid[op], nt = h->ntiles[op], te = h->tile_elems[op];
    switch (op) {
        case kOpPredict: batch_tiles<kOpPredict><<<g, kBlk, 0, st>>>(h->ctl, h->tiles[op], nt, te, h->post_partials); break;
        case kOpBndStar: batch_tiles<kOpBndStar><<<g, kBlk, 0, st>>>(h->ctl, h->tiles[op], nt, te, h->post_partials); break;
        case kOpRhs: batch_tiles<kOpRhs><<<g, kBlk, 0, st>>>(h->ctl, h->tiles[op], nt, te, h->post_partials); break;
        case kOpCorrect: batch_tiles<kOpCorrect><<<g, kBlk, 0, st>>>(h->ctl, h->tiles[op], nt, te, h->post_partials); break;
        case kOpBndNew: batch_tiles<kOpBndNew><<<g, kBlk, 0, st>>>(h->ctl, h->tiles[op], nt, te, h->post_partials); break;
        default: batch_tiles<kOpPost><<<g, kBlk, 0, st>>>(h->ctl, h->tiles[op], nt, te, h->post_partials); break;
    }
    return cudaGetLastError();
}

// (Re)builds the tile table of one op; the post ranges go into the controls.
cudaError_t set_tiles(FlursysBatchHandle *h, int op, int elems) {
    std::vector<int> first;
    std::vector<int2> t = make_tiles(h, op, elems, op == kOpPost ? &first : nullptr);
    if (h->tiles[op]) cudaFree(h->tiles[op]);
    h->tiles[op] = nullptr;
    cudaError_t e = cudaMalloc(&h->tiles[op], sizeof(int2) * std::max<size_t>(t.size(), 1));
    if (e == cudaSuccess) e = cudaMemcpy(h->tiles[op], t.data(), sizeof(int2) * t.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
    h->ntiles[op] = (int)t.size();
    h->tile_elems[op] = elems;
    h->grid[op] = std::max(1, std::min(h->ntiles[op], max_grid(op, h->sms)));
    if (op == kOpPost) {
        if (h->post_partials) cudaFree(h->post_partials);
        h->post_partials = nullptr;
        e = cudaMalloc(&h->post_partials, sizeof(double) * kPostParts * std::max<size_t>(t.size(), 1));
        if (e != cudaSuccess) return e;
        for (int i = 0; i < h->n; ++i) {
            h->h_ctl[i].post_t0 = first[i];
            h->h_ctl[i].post_t1 = first[i + 1];
        }
        e = cudaMemcpy(h->ctl, h->h_ctl.data(), sizeof(BatchCtl) * h->n, cudaMemcpyHostToDevice);
    }
    return e;
}

cudaError_t enqueue_step(FlursysBatchHandle *h, cudaStream_t st) {
    batch_begin<<<1, kBlk, 0, st>>>(h->ctl, h->pin, h->n, h->pcg_blocks);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = launch_op(h, kOpPredict, st);
    if (e == cudaSuccess) e = launch_op(h, kOpBndStar, st);
    if (e == cudaSuccess) e = launch_op(h, kOpRhs, st);
    if (e == cudaSuccess) e = pcg2d_launch(h->pin, h->n, h->pcg_blocks, h->precision, st);
    if (e == cudaSuccess) e = launch_op(h, kOpCorrect, st);
    if (e == cudaSuccess) e = launch_op(h, kOpBndNew, st);
    if (e == cudaSuccess) e = launch_op(h, kOpPost, st);
    if (e == cudaSuccess) {
        batch_end<<<h->n, kBlk, 0, st>>>(h->ctl, h->res, h->post_partials, h->rep, h->dev_err);
        e = cudaGetLastError();
    }
    return e;
}


// Mean device milliseconds of `reps` calls of fn after one warm-up call.
template <typename F>
float time_ms(FlursysBatchHandle *h, int reps, F fn, cudaError_t *e) {
    *e = fn();
    if (*e != cudaSuccess) return 0.f;
    *e = cudaEventRecord(h->ev0, h->stream);
    for (int r = 0; r < reps && *e == cudaSuccess; ++r) *e = fn();
    if (*e == cudaSuccess) *e = cudaEventRecord(h->ev1, h->stream);
    if (*e == cudaSuccess) *e = cudaEventSynchronize(h->ev1);
    float ms = 0.f;
    if (*e == cudaSuccess) *e = cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    return ms / reps;
}

cudaError_t autotune(FlursysBatchHandle *h) {
    cudaError_t e = cudaSuccess;
    // tile kernels: every op is idempotent on the initial state
    static const int kCand[] = {256, 512, 1024, 2048, 4096};
    for (int op = 0; op < kNumOps && e == cudaSuccess; ++op) {
        const bool bnd = op == kOpBndStar || op == kOpBndNew;
        const int ncand = bnd ? 2 : 5;
        int best = kCand[0];
        float best_ms = 1e30f;
        for (int k = 0; k < ncand && e == cudaSuccess; ++k) {
            e = set_tiles(h, op, kCand[k]);
            if (e != cudaSuccess) break;
            const float ms = time_ms(h, 5, [&] { return launch_op(h, op, h->stream); }, &e);
            if (e == cudaSuccess && ms < best_ms) { best_ms = ms; best = kCand[k]; }
        }
        if (e == cudaSuccess) e = set_tiles(h, op, best);
    }
    if (e != cudaSuccess) return e;
    // pressure kernel: blocks per SM on a synthetic right-hand side, with the
    // iteration caps scaled like the expected iteration counts
    std::vector<Pcg2dInstance> tune = h->h_pin;
    for (int i = 0; i < h->n; ++i) {
        const double cells = double(h->h_ctl[i].cells);
        tune[i].max_iters = std::max<long long>(8, (long long)(std::sqrt(cells) / 4.0));
        synth_rhs<<<std::min(1024, (int)((cells + 255) / 256)), 256, 0, h->stream>>>(
            const_cast<double *>(h->h_pin[i].rhs), h->h_pin[i].flags, (int)cells, 0x9E3779B9u + (unsigned)i);
    }
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->pin, tune.data(), sizeof(Pcg2dInstance) * h->n, cudaMemcpyHostToDevice, h->stream);
    int best = h->pcg_per_sm;
    float best_ms = 1e30f;
    for (int per = 1; per <= std::min(h->pcg_max_per_sm, 4) && e == cudaSuccess; ++per) {
        const int blocks = h->sms * per;
        if (blocks < h->n) continue;
        const float ms = time_ms(h, 3, [&] {
            for (int i = 0; i < h->n; ++i) {
                cudaError_t m = cudaMemsetAsync(h->h_pin[i].x, 0, sizeof(double) * h->h_ctl[i].cells, h->stream);
                if (m != cudaSuccess) return m;
            }
            batch_prepare_pressure<<<1, kBlk, 0, h->stream>>>(h->ctl, h->pin, h->n, blocks);
            cudaError_t m = cudaGetLastError();
            if (m == cudaSuccess) m = pcg2d_launch(h->pin, h->n, blocks, h->precision, h->stream);
            return m;
        }, &e);
        if (e == cudaSuccess && ms < best_ms) { best_ms = ms; best = per; }
    }
    h->pcg_per_sm = best;
    h->pcg_blocks = h->sms * best;
    // back to the initial state
    for (int i = 0; i < h->n && e == cudaSuccess; ++i) {
        e = cudaMemsetAsync(h->h_pin[i].x, 0, sizeof(double) * h->h_ctl[i].cells, h->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(const_cast<double *>(h->h_pin[i].rhs), 0, sizeof(double) * h->h_ctl[i].cells, h->stream);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->pin, h->h_pin.data(), sizeof(Pcg2dInstance) * h->n, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    return e;
}

void destroy_handle(FlursysBatchHandle *h) {
    if (!h) return;
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    for (int op = 0; op < kNumOps; ++op)
        if (h->tiles[op]) cudaFree(h->tiles[op]);
    if (h->post_partials) cudaFree(h->post_partials);
    if (h->pool) cudaFree(h->pool);
    if (h->h_rep) cudaFreeHost(h->h_rep);
    if (h->h_ctl_pinned) cudaFreeHost(h->h_ctl_pinned);
    if (h->h_dev_err) cudaFreeHost(h->h_dev_err);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

}  // namespace

extern "C" int32_t flursys_cuda_batch_create(const FlursysCudaConfig *configs, int32_t count, int32_t flags,
                                             FlursysBatchHandle **out) {
    if (!configs || !out || count < 1) return fail("batch: null configs/out or count < 1", FLURSYS_ERR_INVALID_ARGUMENT);
    *out = nullptr;
    if (count > 4096) return fail("batch: at most 4096 instances", FLURSYS_ERR_INVALID_ARGUMENT);
    if (flags & ~(FLURSYS_BATCH_AUTOTUNE | FLURSYS_BATCH_NO_GRAPH)) return fail("batch: unknown flags", FLURSYS_ERR_INVALID_ARGUMENT);
    for (int i = 0; i < count; ++i) {
        const FlursysCudaConfig &c = configs[i];
        std::string msg;
        int32_t st = validate_config_checked(c, &msg);
        char buf[600];
        if (st) {
            std::snprintf(buf, sizeof buf, "batch instance %d: %s", i, msg.c_str());
            return fail(buf, st);
        }
        const char *why = nullptr;
        if (c.dimension != 2) why = "the batched solver is 2D only";
        else if (c.coupling != FLURSYS_COUPLING_PROJECTION) why = "the batched solver supports projection coupling only";
        else if (c.pressure_solver != FLURSYS_PRESSURE_PCG && c.pressure_solver != FLURSYS_PRESSURE_SOR) why = "the batched solver supports the PCG and SOR pressure solvers";
        else if (c.physics.energy_model != FLURSYS_ENERGY_OFF) why = "the batched solver runs constant-property flow only; thermal and buoyancy models are not available";
        else if (c.precision != configs[0].precision) why = "every instance must use the same precision";
        else if (c.device != configs[0].device) why = "every instance must use the same device";
        if (why) {
            std::snprintf(buf, sizeof buf, "batch instance %d: %s", i, why);
            return fail(buf, FLURSYS_ERR_UNSUPPORTED);
        }
        if ((long long)(c.nx + 1) * (c.ny + 1) >= (1LL << 30)) {
            std::snprintf(buf, sizeof buf, "batch instance %d: grid too large", i);
            return fail(buf, FLURSYS_ERR_INVALID_CONFIG);
        }
    }
    auto *h = new FlursysBatchHandle();
    h->n = count;
    h->precision = configs[0].precision;
    h->device = configs[0].device;
    h->use_graph = !(flags & FLURSYS_BATCH_NO_GRAPH);
    cudaError_t e = cudaSetDevice(h->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device);
    int coop = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, h->device);
    if (e == cudaSuccess && !coop) { destroy_handle(h); return fail("batch: device does not support cooperative launches", FLURSYS_ERR_UNSUPPORTED); }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&h->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&h->ev1);
    int maxgrid = 0;
    if (e == cudaSuccess) e = pcg2d_max_grid(h->precision, h->device, &maxgrid);
    if (e != cudaSuccess) { destroy_handle(h); return cuda_fail(e, "batch create"); }
    h->pcg_max_per_sm = std::max(1, maxgrid / h->sms);
    h->pcg_per_sm = h->pcg_max_per_sm;
    h->pcg_blocks = h->sms * h->pcg_per_sm;
    if (h->pcg_blocks < count) { destroy_handle(h); return fail("batch: more instances than co-resident pressure blocks", FLURSYS_ERR_INVALID_ARGUMENT); }

    // host case data and the pooled device layout
    const size_t vsize = h->precision == FLURSYS_PRECISION_MIXED ? 4 : 8;
    std::vector<Case2dHost> cases(count);
    struct Offs { size_t f[13], bnd[8], flags, work[5], partials, barrier, diag; };
    std::vector<Offs> off(count);
    size_t pos = 0;
    auto take = [&](size_t bytes) { const size_t at = pos; pos += align_up(std::max<size_t>(bytes, 1)); return at; };
    h->nx.resize(count);
    h->ny.resize(count);
    for (int i = 0; i < count; ++i) {
        build_case2d(configs[i], &cases[i]);
        const int nx = (int)configs[i].nx, ny = (int)configs[i].ny;
        h->nx[i] = nx;
        h->ny[i] = ny;
        const size_t nc = (size_t)nx * ny, nu = (size_t)(nx + 1) * ny, nv = (size_t)nx * (ny + 1);
        const size_t sizes[13] = {nu, nv, nu, nv, nu, nv, nc, nc, nc, nc, nc, nc, nc};
        for (int k = 0; k < 13; ++k) off[i].f[k] = take(8 * sizes[k]);
        for (int k = 0; k < 8; ++k) off[i].bnd[k] = take(8 * cases[i].bnd[k].size());
        off[i].flags = take(nc);
        for (int k = 0; k < 5; ++k) off[i].work[k] = take(vsize * nc);
        const size_t cap = std::min<size_t>((size_t)h->pcg_blocks, (nc + kBlk - 1) / kBlk);
        off[i].partials = take(8 * cap * pcg2d_num_partials());
        off[i].barrier = take(sizeof(GridBarrier));
        off[i].diag = take(sizeof(Diag2Dev));
    }
    const size_t ctl_off = take(sizeof(BatchCtl) * count);
    const size_t pin_off = take(sizeof(Pcg2dInstance) * count);
    const size_t res_off = take(sizeof(PcgResultDev) * count);
    const size_t rep_off = take(sizeof(FlursysStepReport) * count);
    const size_t err_off = take(sizeof(unsigned));
    h->pool_bytes = pos;
    e = cudaMalloc(&h->pool, pos);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->pool, 0, pos, h->stream);
    if (e == cudaSuccess) e = cudaMallocHost(&h->h_rep, sizeof(FlursysStepReport) * count);
    if (e == cudaSuccess) e = cudaMallocHost(&h->h_ctl_pinned, sizeof(BatchCtl) * count);
    if (e == cudaSuccess) e = cudaMallocHost(&h->h_dev_err, sizeof(unsigned));
    if (e != cudaSuccess) { destroy_handle(h); return cuda_fail(e, "batch allocation"); }
    char *P = h->pool;
    h->ctl = reinterpret_cast<BatchCtl *>(P + ctl_off);
    h->pin = reinterpret_cast<Pcg2dInstance *>(P + pin_off);
    h->res = reinterpret_cast<PcgResultDev *>(P + res_off);
    h->rep = reinterpret_cast<FlursysStepReport *>(P + rep_off);
    h->dev_err = reinterpret_cast<unsigned *>(P + err_off);
    h->h_ctl.assign(count, BatchCtl{});
    h->h_pin.assign(count, Pcg2dInstance{});
    for (int i = 0; i < count && e == cudaSuccess; ++i) {
        const FlursysCudaConfig &c = configs[i];
        const Case2dHost &cs = cases[i];
        const Offs &o = off[i];
        BatchCtl &b = h->h_ctl[i];
        Cavity2dState &s = b.s;
        const int nx = h->nx[i], ny = h->ny[i];
        const size_t nc = (size_t)nx * ny;
        s.nx = nx; s.ny = ny; s.sms = h->sms;
        s.dx = c.case_params.length / nx;
        s.dy = c.case_params.height / ny;
        s.rho = c.case_params.density;
        s.nu = c.case_params.kinematic_viscosity;
        s.convection = c.convection;
        for (int side = 0; side < 4; ++side) s.kind[side] = cs.kind[side];
        s.flags = reinterpret_cast<const uint8_t *>(P + o.flags);
        double *bd[8];
        for (int k = 0; k < 8; ++k) bd[k] = reinterpret_cast<double *>(P + o.bnd[k]);
        s.bu_left = bd[0]; s.bu_right = bd[1]; s.bv_bottom = bd[2]; s.bv_top = bd[3];
        s.gu_bottom = bd[4]; s.gu_top = bd[5]; s.gv_left = bd[6]; s.gv_right = bd[7];
        double *f[13];
        for (int k = 0; k < 13; ++k) f[k] = reinterpret_cast<double *>(P + o.f[k]);
        s.u = f[0]; s.v = f[1]; s.un = f[2]; s.vn = f[3]; s.us = f[4]; s.vs = f[5];
        s.p = f[6]; s.rhs = f[7]; s.pold = f[8];
        s.uc = f[9]; s.vc = f[10]; s.speed = f[11]; s.vort = f[12];
        s.cylinder = c.case_params.kind == FLURSYS_CASE_CYLINDER;
        s.cylinder_mu = c.case_params.cylinder_mu;
        s.partials = nullptr;
        s.post_blocks = 0;
        s.diag = reinterpret_cast<Diag2Dev *>(P + o.diag);
        b.dt_cfg = c.dt; b.min_dt = c.min_dt; b.max_dt = c.max_dt;
        b.target_cfl = c.target_cfl; b.target_diff = c.target_diffusion_number; b.max_growth = c.max_growth_factor;
        b.t_end = c.t_end;
        b.steady_tol = c.steady_tolerance;
        b.pressure_tol = c.pressure_tolerance;
        const FlursysCaseParams &cp = c.case_params;
        b.force_q = 0.5 * cp.density * cp.reference_velocity * cp.reference_velocity * cp.cylinder_diameter;
        b.minimum_steps = c.minimum_steps;
        b.adaptive = c.adaptive ? 1 : 0;
        b.case_kind = cp.kind;
        b.current_dt = c.dt; b.time = 0.0; b.step_dt = c.dt;
        b.max_u = cs.max_u; b.max_v = cs.max_v;
        b.step = 0; b.last_iters = 0;
        b.active = 1; b.status = FLURSYS_OK;
        b.cells = (long long)nc;
        Pcg2dInstance &in = h->h_pin[i];
        in.nx = nx; in.ny = ny;
        in.idx2 = 1.0 / (s.dx * s.dx);
        in.idy2 = 1.0 / (s.dy * s.dy);
        in.flags = s.flags;
        in.x = s.p;
        in.rhs = s.rhs;
        void *w[5];
        for (int k = 0; k < 5; ++k) w[k] = P + o.work[k];
        in.r = w[0]; in.z = w[1]; in.d0 = w[2]; in.d1 = w[3]; in.q = w[4];
        in.outlet_pressure = cs.outlet_p;
        in.project = cs.project ? 1 : 0;
        in.ref_cell = cs.ref_cell;
        in.count_fluid = cs.fluid;
        in.block0 = 0; in.nblocks = 0;
        in.partials = reinterpret_cast<double *>(P + o.partials);
        in.barrier = reinterpret_cast<GridBarrier *>(P + o.barrier);
        in.result = h->res + i;
        in.solver = c.pressure_solver == FLURSYS_PRESSURE_SOR ? FLURSYS_PRESSURE_SOR : FLURSYS_PRESSURE_PCG;
        in.stop_rule = c.stop_rule == FLURSYS_STOP_REL_L2 ? FLURSYS_STOP_REL_L2 : FLURSYS_STOP_ABS_INF;
        in.tol = c.pressure_tolerance;
        in.atol = c.pressure_atol;
        in.rtol = c.pressure_rtol;
        in.omega = c.pressure_omega;
        in.max_iters = c.pressure_max_iters;
        in.replace_every = c.residual_replacement_every > 0 ? c.residual_replacement_every : 50;
        // case data
        e = cudaMemcpyAsync(P + o.flags, cs.flags.data(), nc, cudaMemcpyHostToDevice, h->stream);
        for (int k = 0; k < 8 && e == cudaSuccess; ++k)
            e = cudaMemcpyAsync(bd[k], cs.bnd[k].data(), 8 * cs.bnd[k].size(), cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(s.u, cs.u.data(), 8 * cs.u.size(), cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(s.v, cs.v.data(), 8 * cs.v.size(), cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);  // the host vectors of this case go out of scope later
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->ctl, h->h_ctl.data(), sizeof(BatchCtl) * count, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->pin, h->h_pin.data(), sizeof(Pcg2dInstance) * count, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    static const int kDefaultTile[kNumOps] = {1024, 256, 1024, 1024, 256, 1024};
    for (int op = 0; op < kNumOps && e == cudaSuccess; ++op) e = set_tiles(h, op, kDefaultTile[op]);
    if (e != cudaSuccess) { destroy_handle(h); return cuda_fail(e, "batch set-up"); }
    if (flags & FLURSYS_BATCH_AUTOTUNE) {
        const auto t0 = std::chrono::steady_clock::now();
        e = autotune(h);
        h->tune_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (e != cudaSuccess) { destroy_handle(h); return cuda_fail(e, "batch autotune"); }
    }
    if (h->use_graph) {
        e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t ce = enqueue_step(h, h->stream);
            e = cudaStreamEndCapture(h->stream, &h->graph);
            if (ce != cudaSuccess) e = ce;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&h->exec, h->graph, 0);
        size_t nodes = 0;
        if (e == cudaSuccess) e = cudaGraphGetNodes(h->graph, nullptr, &nodes);
        h->graph_nodes = (int)nodes;
        if (e != cudaSuccess) { destroy_handle(h); return cuda_fail(e, "batch step graph"); }
    }
    *out = h;
    return FLURSYS_OK;
}

extern "C" int32_t flursys_cuda_batch_step(FlursysBatchHandle *h, int64_t nsteps) {
    if (!h) return fail("batch: null handle", FLURSYS_ERR_INVALID_ARGUMENT);
    if (nsteps < 0) return fail("batch: nsteps must be non-negative", FLURSYS_ERR_INVALID_ARGUMENT);
    if (nsteps == 0) return FLURSYS_OK;
    cudaError_t e = cudaSetDevice(h->device);
    if (e == cudaSuccess) e = cudaEventRecord(h->ev0, h->stream);
    for (int64_t k = 0; k < nsteps && e == cudaSuccess; ++k)
        e = h->use_graph ? cudaGraphLaunch(h->exec, h->stream) : enqueue_step(h, h->stream);
    if (e == cudaSuccess) e = cudaEventRecord(h->ev1, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->h_dev_err, h->dev_err, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "batch step");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->last_step_ms = double(ms) / double(nsteps);
    if (*h->h_dev_err & kDevErrBarrierTimeout)
        return fail("batch: a pressure-solver grid barrier timed out", FLURSYS_ERR_TIMEOUT);
    return FLURSYS_OK;
}

extern "C" int32_t flursys_cuda_batch_report(FlursysBatchHandle *h, int32_t instance, FlursysStepReport *report,
                                             int32_t *instance_status) {
    if (!h || !report) return fail("batch: null handle or report", FLURSYS_ERR_INVALID_ARGUMENT);
    if (instance < 0 || instance >= h->n) return fail("batch: instance out of range", FLURSYS_ERR_INVALID_ARGUMENT);
    cudaError_t e = cudaSetDevice(h->device);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->h_rep + instance, h->rep + instance, sizeof(FlursysStepReport), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->h_ctl_pinned + instance, h->ctl + instance, sizeof(BatchCtl), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "batch report");
    *report = h->h_rep[instance];
    report->step_ms = h->last_step_ms;
    if (instance_status) *instance_status = h->h_ctl_pinned[instance].active ? FLURSYS_OK : h->h_ctl_pinned[instance].status;
    return FLURSYS_OK;
}

extern "C" int32_t flursys_cuda_batch_download(FlursysBatchHandle *h, int32_t instance, int32_t field_id, double *host,
                                               size_t n) {
    if (!h || !host) return fail("batch: null handle or buffer", FLURSYS_ERR_INVALID_ARGUMENT);
    if (instance < 0 || instance >= h->n) return fail("batch: instance out of range", FLURSYS_ERR_INVALID_ARGUMENT);
    cudaError_t e = cudaSetDevice(h->device);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->h_ctl_pinned + instance, h->ctl + instance, sizeof(BatchCtl), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "batch download");
    const Cavity2dState &s = h->h_ctl_pinned[instance].s;
    const size_t nc = (size_t)s.nx * s.ny, nu = (size_t)(s.nx + 1) * s.ny, nv = (size_t)s.nx * (s.ny + 1);
    const double *p = nullptr;
    size_t m = 0;
    switch (field_id) {
        case FLURSYS_FIELD_U: p = s.u; m = nu; break;
        case FLURSYS_FIELD_V: p = s.v; m = nv; break;
        case FLURSYS_FIELD_PRESSURE: p = s.p; m = nc; break;
        case FLURSYS_FIELD_RHS: p = s.rhs; m = nc; break;
        case FLURSYS_FIELD_U_STAR: p = s.us; m = nu; break;
        case FLURSYS_FIELD_V_STAR: p = s.vs; m = nv; break;
        case FLURSYS_FIELD_SPEED: p = s.speed; m = nc; break;
        case FLURSYS_FIELD_VORTICITY: p = s.vort; m = nc; break;
        case FLURSYS_FIELD_U_CELL: p = s.uc; m = nc; break;
        case FLURSYS_FIELD_V_CELL: p = s.vc; m = nc; break;
        default: return fail("batch: field not available for a 2D instance", FLURSYS_ERR_INVALID_ARGUMENT);
    }
    if (n != m) {
        char buf[160];
        std::snprintf(buf, sizeof buf, "batch: field %d of instance %d has %zu values, buffer has %zu", field_id, instance, m, n);
        return fail(buf, FLURSYS_ERR_INVALID_ARGUMENT);
    }
    e = cudaMemcpyAsync(host, p, sizeof(double) * m, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "batch download");
    return FLURSYS_OK;
}

extern "C" int32_t flursys_cuda_batch_tuning(const FlursysBatchHandle *h, FlursysBatchTuning *out) {
    if (!h || !out) return fail("batch: null handle or output", FLURSYS_ERR_INVALID_ARGUMENT);
    std::memset(out, 0, sizeof *out);
    for (int op = 0; op < kNumOps; ++op) out->tile_elems[op] = h->tile_elems[op];
    out->pressure_blocks_per_sm = h->pcg_per_sm;
    out->pressure_blocks = h->pcg_blocks;
    out->graph_nodes = h->graph_nodes;
    out->tune_ms = h->tune_ms;
    return FLURSYS_OK;
}

extern "C" int32_t flursys_cuda_batch_destroy(FlursysBatchHandle *h) {
    if (!h) return FLURSYS_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    destroy_handle(h);
    return FLURSYS_OK;
}
