// pcg3d.cu — persistent Jacobi-PCG for the pinned 7-point pressure system of
// the 3D lid-driven cavity (sm_100a).
//
// System: the one the reference's 3D SOR converges to
// (src/solver/incompressible_3d.rs:293-332, pressure_neighbor :450-474):
// for every cell c != (0,0,0),  sum_{in-range nb} w (p_c - p_nb) = -rhs_c,
// with p_(0,0,0) = 0 (w = 1/dx^2, 1/dy^2, 1/dz^2). Out-of-range neighbours
// drop out (Neumann walls). Cell (0,0,0) is an identity row.
//
// Iteration order follows solve_pressure_pcg (src/solver/incompressible.rs:
// 1125-1186): q = A d; alpha = rz/dq; x += alpha d; r -= alpha q; stop test;
// z = r/diag; rz_new; beta; d = z + beta d. The direction update is fused into
// the next stencil pass: each pass forms d_new = z + beta d_old on the fly for
// its cells and their halo (bit-identical in every block) and writes d_new
// into the other half of a double buffer.
//
// One cooperative launch runs the whole solve. Two bounded grid barriers per
// iteration separate the reductions (d.q, then r.r / r.z / max|r|); every
// block reduces the per-block partials itself in a fixed order, so all blocks
// take bit-identical decisions and leave the loop together.
//
// Precision modes:
//   F64   — r, d, q in FP64; x (= p) updated in place. Parity mode.
//   MIXED — r, d, q in FP32 and the stencil in FP32; dots, norms and alpha/beta
//           in FP64; the solution increment accumulates in an FP32 buffer that
//           is folded into the FP64 pressure every `replace_every` iterations,
//           when the FP32 residual is replaced by the FP64 true residual
//           b - A x. Convergence is accepted only after such a replacement, so
//           the stop test always holds for the FP64 true residual.
#include <cuda_runtime.h>

#include <cmath>

#include "common.cuh"
#include "pcg3d.cuh"

namespace flursys {

namespace {

constexpr int kBlock = 256;
constexpr int kNumPartials = 4;  // slot 0: d.q ; slots 0..2: r.r, r.z, max|r|

struct Geo3 {
    int nx, ny, nz;
    long long nxy, n;
    double ix2, iy2, iz2;
};

__device__ __forceinline__ double diag3(const Geo3 &g, int i, int j, int k) {
    double d = 0.0;
    d += (i > 0) ? g.ix2 : 0.0;
    d += (i + 1 < g.nx) ? g.ix2 : 0.0;
    d += (j > 0) ? g.iy2 : 0.0;
    d += (j + 1 < g.ny) ? g.iy2 : 0.0;
    d += (k > 0) ? g.iz2 : 0.0;
    d += (k + 1 < g.nz) ? g.iz2 : 0.0;
    return d;
}

// z = r / diag, identity on the pinned cell.
template <typename V>
__device__ __forceinline__ V zval(const Geo3 &g, const V *__restrict__ r, long long c, int i, int j,
                                  int k) {
    if (c == 0) return V(0);
    return V(double(__ldcg(r + c)) / diag3(g, i, j, k));
}

// d_new = z + beta * d_old at cell c; d_old is not read on the first pass.
template <typename V>
__device__ __forceinline__ V dnew(const Geo3 &g, const V *__restrict__ r, const V *__restrict__ dold,
                                  double beta, bool first, long long c, int i, int j, int k) {
    if (c == 0) return V(0);
    V z = zval<V>(g, r, c, i, j, k);
    if (first) return z;
    return V(double(z) + beta * double(__ldcg(dold + c)));
}

// Residual of the FP64 system at cell c: b_c - (A x)_c with b = -rhs.
__device__ __forceinline__ double true_residual(const Geo3 &g, const double *__restrict__ x,
                                                const double *__restrict__ rhs, long long c, int i,
                                                int j, int k) {
    if (c == 0) return 0.0;
    const double xc = __ldcg(x + c);
    double dg = 0.0, s = 0.0;
    if (i > 0) { dg += g.ix2; s += (c - 1 == 0) ? 0.0 : g.ix2 * __ldcg(x + c - 1); }
    if (i + 1 < g.nx) { dg += g.ix2; s += g.ix2 * __ldcg(x + c + 1); }
    if (j > 0) { dg += g.iy2; s += (c - g.nx == 0) ? 0.0 : g.iy2 * __ldcg(x + c - g.nx); }
    if (j + 1 < g.ny) { dg += g.iy2; s += g.iy2 * __ldcg(x + c + g.nx); }
    if (k > 0) { dg += g.iz2; s += (c - g.nxy == 0) ? 0.0 : g.iz2 * __ldcg(x + c - g.nxy); }
    if (k + 1 < g.nz) { dg += g.iz2; s += g.iz2 * __ldcg(x + c + g.nxy); }
    return -__ldcg(rhs + c) - (dg * xc - s);
}

__device__ __forceinline__ void decode(const Geo3 &g, long long c, int &i, int &j, int &k) {
    k = int(c / g.nxy);
    long long rem = c - (long long)k * g.nxy;
    j = int(rem / g.nx);
    i = int(rem - (long long)j * g.nx);
}

template <typename V, bool MIXED>
__global__ void __launch_bounds__(kBlock) pcg3d_kernel(Pcg3dArgs a) {
    __shared__ double s_red[kBlock / 32];
    const Geo3 g{a.nx, a.ny, a.nz, (long long)a.nx * a.ny, (long long)a.nx * a.ny * a.nz,
                 a.ix2, a.iy2, a.iz2};
    const long long stride = (long long)gridDim.x * kBlock;
    const long long tid0 = (long long)blockIdx.x * kBlock + threadIdx.x;
    double *x = a.x;
    const double *rhs = a.rhs;
    V *r = static_cast<V *>(a.r);
    V *dbuf[2] = {static_cast<V *>(a.d0), static_cast<V *>(a.d1)};
    V *q = static_cast<V *>(a.q);
    float *dx = a.dx;  // MIXED only
    double *part = a.partials;
    GridBarrier *bar = a.barrier;
    const bool l2 = a.stop_rule == FLURSYS_STOP_REL_L2;

    // ---- r = b - A x (FP64), z = r/diag, partial r.r, r.z, max|r| ----
    auto residual_pass = [&](bool zero_dx) {
        double srr = 0.0, srz = 0.0, smax = 0.0;
        for (long long c = tid0; c < g.n; c += stride) {
            int i, j, k;
            decode(g, c, i, j, k);
            double rr = true_residual(g, x, rhs, c, i, j, k);
            V rv = V(rr);
            r[c] = rv;
            if (MIXED && zero_dx) dx[c] = 0.f;
            double rd = double(rv);
            double z = (c == 0) ? rd : rd / diag3(g, i, j, k);
            srr += rd * rd;
            srz += rd * z;
            smax = fmax(smax, fabs(rd));
        }
        double t0 = block_sum<kBlock>(srr, s_red);
        double t1 = block_sum<kBlock>(srz, s_red);
        double t2 = block_max<kBlock>(smax, s_red);
        if (threadIdx.x == 0) {
            part[blockIdx.x * kNumPartials + 0] = t0;
            part[blockIdx.x * kNumPartials + 1] = t1;
            part[blockIdx.x * kNumPartials + 2] = t2;
        }
    };
    auto reduce3 = [&](double &rr, double &rz, double &rmax) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += kBlock) {
            s0 += __ldcg(&part[b * kNumPartials + 0]);
            s1 += __ldcg(&part[b * kNumPartials + 1]);
            s2 = fmax(s2, __ldcg(&part[b * kNumPartials + 2]));
        }
        rr = block_sum<kBlock>(s0, s_red);
        rz = block_sum<kBlock>(s1, s_red);
        rmax = block_max<kBlock>(s2, s_red);
    };
    // Folds the FP32 increment into the FP64 solution (MIXED).
    auto fold = [&]() {
        for (long long c = tid0; c < g.n; c += stride) {
            if (c == 0) { x[0] = 0.0; continue; }
            x[c] += double(__ldcg(dx + c));
        }
    };

    int status = FLURSYS_LINEAR_MAX_ITERATIONS;
    int error = 0;  // FlursysStatus of a failure
    long long iterations = 0;
    double residual = 0.0, initial = 0.0, threshold = 0.0;

    if (blockIdx.x == 0 && threadIdx.x == 0) x[0] = 0.0;
    // x[0] is read as the pinned value 0 by every stencil, so no barrier is
    // needed before the first residual pass.
    residual_pass(true);
    if (!grid_sync(bar)) return;
    double rr, rz_old, rmax;
    reduce3(rr, rz_old, rmax);
    const double initial_l2 = sqrt(rr);
    initial = l2 ? initial_l2 : rmax;
    threshold = l2 ? a.atol + a.rtol * initial : a.tol;
    residual = initial;
    bool done = l2 ? (residual <= threshold) : (residual < threshold);
    if (done) status = FLURSYS_LINEAR_CONVERGED;
    double beta = 0.0;
    bool first = true;

    for (long long it = 0; !done && it < a.max_iters; ++it) {
        iterations = it + 1;
        V *dcur = dbuf[it & 1];
        const V *dold = dbuf[(it + 1) & 1];
        // ---- phase A: d = z + beta d_old (cells + halo), q = A d, partial d.q ----
        double sdq = 0.0;
        for (long long c = tid0; c < g.n; c += stride) {
            int i, j, k;
            decode(g, c, i, j, k);
            V dc = dnew<V>(g, r, dold, beta, first, c, i, j, k);
            V qc;
            if (c == 0) {
                qc = dc;
            } else {
                const V wx = V(g.ix2), wy = V(g.iy2), wz = V(g.iz2);
                V dg = V(0), s = V(0);
                if (i > 0) { dg += wx; if (c - 1 != 0) s += wx * dnew<V>(g, r, dold, beta, first, c - 1, i - 1, j, k); }
                if (i + 1 < g.nx) { dg += wx; s += wx * dnew<V>(g, r, dold, beta, first, c + 1, i + 1, j, k); }
                if (j > 0) { dg += wy; if (c - g.nx != 0) s += wy * dnew<V>(g, r, dold, beta, first, c - g.nx, i, j - 1, k); }
                if (j + 1 < g.ny) { dg += wy; s += wy * dnew<V>(g, r, dold, beta, first, c + g.nx, i, j + 1, k); }
                if (k > 0) { dg += wz; if (c - g.nxy != 0) s += wz * dnew<V>(g, r, dold, beta, first, c - g.nxy, i, j, k - 1); }
                if (k + 1 < g.nz) { dg += wz; s += wz * dnew<V>(g, r, dold, beta, first, c + g.nxy, i, j, k + 1); }
                qc = dg * dc - s;
            }
            dcur[c] = dc;
            q[c] = qc;
            sdq += double(dc) * double(qc);
        }
        {
            double t = block_sum<kBlock>(sdq, s_red);
            if (threadIdx.x == 0) part[blockIdx.x * kNumPartials + 3] = t;
        }
        if (!grid_sync(bar)) return;
        double dq;
        {
            double s = 0.0;
            for (int b = threadIdx.x; b < (int)gridDim.x; b += kBlock) s += __ldcg(&part[b * kNumPartials + 3]);
            dq = block_sum<kBlock>(s, s_red);
        }
        if (fabs(dq) < 1.0e-30 || !isfinite(dq)) { error = FLURSYS_ERR_BREAKDOWN; break; }
        const double alpha = rz_old / dq;
        if (!isfinite(alpha)) { error = FLURSYS_ERR_BREAKDOWN; break; }
        // ---- phase B: x += alpha d, r -= alpha q, partial r.r, r.z, max|r| ----
        double srr = 0.0, srz = 0.0, smax = 0.0;
        for (long long c = tid0; c < g.n; c += stride) {
            const double dc = double(dcur[c]);
            const double qc = double(__ldcg(q + c));
            if (MIXED) {
                dx[c] = float(double(__ldcg(dx + c)) + alpha * dc);
            } else {
                if (c != 0) x[c] = __ldcg(x + c) + alpha * dc;
            }
            const V rv = V(double(__ldcg(r + c)) - alpha * qc);
            r[c] = rv;
            const double rd = double(rv);
            double z = rd;
            if (c != 0) {
                int i, j, k;
                decode(g, c, i, j, k);
                z = rd / diag3(g, i, j, k);
            }
            srr += rd * rd;
            srz += rd * z;
            smax = fmax(smax, fabs(rd));
        }
        {
            double t0 = block_sum<kBlock>(srr, s_red);
            double t1 = block_sum<kBlock>(srz, s_red);
            double t2 = block_max<kBlock>(smax, s_red);
            if (threadIdx.x == 0) {
                part[blockIdx.x * kNumPartials + 0] = t0;
                part[blockIdx.x * kNumPartials + 1] = t1;
                part[blockIdx.x * kNumPartials + 2] = t2;
            }
        }
        if (!grid_sync(bar)) return;
        double rz_new;
        reduce3(rr, rz_new, rmax);
        residual = l2 ? sqrt(rr) : rmax;
        if (!isfinite(residual)) { error = FLURSYS_ERR_NON_FINITE; break; }
        bool conv = l2 ? (residual <= threshold) : (residual < threshold);
        if (MIXED && (conv || ((it + 1) % a.replace_every) == 0)) {
            // FP64 residual replacement: fold the increment, recompute r = b - A x.
            fold();
            if (!grid_sync(bar)) return;
            residual_pass(true);
            if (!grid_sync(bar)) return;
            reduce3(rr, rz_new, rmax);
            residual = l2 ? sqrt(rr) : rmax;
            if (!isfinite(residual)) { error = FLURSYS_ERR_NON_FINITE; break; }
            conv = l2 ? (residual <= threshold) : (residual < threshold);
        }
        if (conv) { status = FLURSYS_LINEAR_CONVERGED; break; }
        if (fabs(rz_old) < 1.0e-30) break;
        beta = rz_new / rz_old;
        rz_old = rz_new;
        first = false;
    }

    if (MIXED && error == 0 && status != FLURSYS_LINEAR_CONVERGED) {
        // Leaving at the iteration limit: fold the pending increment.
        fold();
    }
    if (!grid_sync(bar)) return;
    // ---- final FP64 check: ||b - A x||_2 on the solution in HBM ----
    double s_true = 0.0;
    for (long long c = tid0; c < g.n; c += stride) {
        int i, j, k;
        decode(g, c, i, j, k);
        double t = true_residual(g, x, rhs, c, i, j, k);
        s_true += t * t;
    }
    {
        double t = block_sum<kBlock>(s_true, s_red);
        if (threadIdx.x == 0) part[blockIdx.x * kNumPartials + 3] = t;
    }
    if (!grid_sync(bar)) return;
    double true_rr;
    {
        double s = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += kBlock) s += __ldcg(&part[b * kNumPartials + 3]);
        true_rr = block_sum<kBlock>(s, s_red);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        PcgResultDev *res = a.result;
        res->error = error;
        res->status = status;
        res->iterations = iterations;
        res->initial = initial;
        res->residual = residual;
        res->true_l2 = sqrt(true_rr);
        res->initial_l2 = initial_l2;
        res->device_error = bar->error;
    }
}

}  // namespace

size_t pcg3d_vector_bytes(int precision) {
    return precision == FLURSYS_PRECISION_MIXED ? sizeof(float) : sizeof(double);
}

cudaError_t pcg3d_max_grid(int precision, int device, int *grid) {
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    if (precision == FLURSYS_PRECISION_MIXED)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg3d_kernel<float, true>, kBlock, 0);
    else
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg3d_kernel<double, false>, kBlock, 0);
    if (e != cudaSuccess) return e;
    *grid = sms * per_sm;
    return cudaSuccess;
}

int pcg3d_block_size() { return kBlock; }
int pcg3d_num_partials() { return kNumPartials; }

cudaError_t pcg3d_launch(const Pcg3dArgs &args, int grid, int precision, cudaStream_t stream) {
    Pcg3dArgs a = args;
    void *params[] = {&a};
    if (precision == FLURSYS_PRECISION_MIXED)
        return cudaLaunchCooperativeKernel((const void *)pcg3d_kernel<float, true>, dim3(grid), dim3(kBlock),
                                           params, 0, stream);
    return cudaLaunchCooperativeKernel((const void *)pcg3d_kernel<double, false>, dim3(grid), dim3(kBlock),
                                       params, 0, stream);
}

}  // namespace flursys
