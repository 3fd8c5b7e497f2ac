// fcg3d.cu — flexible CG with the learned preconditioner (fcgnet.cuh) for the
// pinned 7-point pressure system of the 3D cavity (the system of pcg3d.cu:
// sum_nb w (p_c - p_nb) = -rhs_c for c != (0,0,0), p_(0,0,0) = 0).
//
// The iteration runs on the equivalent compatible pure-Neumann form A~ x = b~
// (row 0 the ordinary Neumann row with b~_0 = -sum_{c != 0} b_c, so every
// column and b~ sum to zero); its solutions differ from the pinned one by a
// constant, removed at the end by x -= x_0. Unlike the pinned matrix, A~ has
// no tiny eigenvalue tied to the pin, and the network never has to produce
// the pin's global offset. Directions are kept mean-free.
//
// FCG(m) (Notay, "Flexible conjugate gradients", SIAM J. Sci. Comput. 22,
// 2000: truncated A-orthogonalisation against the last m directions, m = 8):
//   z = M(r);  d = z - sum_j (z.q_j)/(d_j.q_j) d_j
//   q = A d;   alpha = (d.r)/(d.q);  x += alpha d;  r -= alpha q
// With one stored direction (m = 1) a preconditioner that is not symmetric
// lets the directions cycle (beta -> -1, alpha -> 0); more stored
// directions keep the search A-orthogonal.
// M is one two-level cycle: damped-Jacobi pre-smoothing (omega 0.8), the
// network on the smoothed residual (its input normalised to unit RMS, output
// scaled by h^2 / scale) as the coarse correction, and damped-Jacobi
// post-smoothing; the smoother takes the rough error modes that the network's
// local receptive field cannot. The first step is the network's initial guess,
// scaled by the A-optimal alpha. Precision as in the mixed PCG: r, z, d, q
// and the stencil in FP32, x and every dot in FP64, the FP32 residual replaced
// by the FP64 true residual b - A x every 50 iterations, whenever it has
// fallen 1000-fold since the last replacement, and before the stop test is
// accepted, so ||b - A x||_2 <= atol + rtol ||b - A x0||_2 holds for the FP64
// solution exactly as for the plain PCG.
//
// Fallback: when the residual has not halved over 25 iterations, a search
// direction breaks down, or the FCG iteration cap is reached, the plain
// Jacobi-PCG (pcg3d.cu) finishes the solve from the current x with the same
// absolute threshold.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "capi_internal.cuh"
#include "common.cuh"
#include "fcgnet.cuh"
#include "flursys_cuda.h"

namespace flursys {

namespace {

constexpr int kBX = 32, kBY = 8;
constexpr int kPw = 256;           // pointwise block
constexpr int kMaxPwBlocks = 1184;
constexpr int kMaxM = 8;           // stored directions of FCG(m), at most
constexpr int kDefaultM = 8;       // and by default
constexpr int kDotStride = kMaxM + 2;  // partials per block of the direction dots

struct FcgScalars {
    double dq, dr, rr, alpha;
    double zmean;         // mean of z (the direction is mean-free)
    double rhs_sum;       // sum of rhs over the cells other than 0
    double x0;            // x at cell 0 before the final shift
    double dqs[kMaxM];    // d_j . q_j of the stored directions, by slot
    double coef[kMaxM];   // (z . q_j) / (d_j . q_j) of the current z, by position
    int breakdown;
    int pad;
};

// The stored directions d_j and q_j = A~ d_j an iteration orthogonalises
// against (positions 0..count-1, in ring slots slot[]).
struct DirSet {
    const float *d[kMaxM];
    const float *q[kMaxM];
    int slot[kMaxM];
    int count;
};

struct Geo3 {
    int nx, ny, nz;
    float wx, wy, wz;       // FP32 stencil weights
    double wxd, wyd, wzd;   // FP64 stencil weights
};

// Off-diagonal sum and diagonal of the pinned operator at (i, j, k) != 0.
template <typename T, typename F>
__device__ __forceinline__ T apply7(const Geo3 &g, int i, int j, int k, T wx, T wy, T wz, T vc, F val) {
    T dg = T(0), s = T(0);
    if (i > 0) { dg += wx; s += wx * val(-1, 0, 0); }
    if (i + 1 < g.nx) { dg += wx; s += wx * val(1, 0, 0); }
    if (j > 0) { dg += wy; s += wy * val(0, -1, 0); }
    if (j + 1 < g.ny) { dg += wy; s += wy * val(0, 1, 0); }
    if (k > 0) { dg += wz; s += wz * val(0, 0, -1); }
    if (k + 1 < g.nz) { dg += wz; s += wz * val(0, 0, 1); }
    return dg * vc - s;
}

__device__ __forceinline__ void write_partials(double *partials, int nblk_index, const double *v, int nv) {
    __shared__ double red[kBX * kBY / 32];
    for (int p = 0; p < nv; ++p) {
        const double t = block_sum<kBX * kBY>(v[p], red);
        if (threadIdx.x == 0) partials[(long long)nblk_index * 2 + p] = t;
    }
}

// r = b - A x in FP64 (b = -rhs; row 0: r = 0), stored in FP32; partial r.r.
__global__ void __launch_bounds__(kBX * kBY) fcg_residual(Geo3 g, const double *__restrict__ x,
                                                          const double *__restrict__ rhs, float *r, double *partials) {
    const int i = blockIdx.x * kBX + (threadIdx.x & 31), j = blockIdx.y * kBY + (threadIdx.x >> 5), k = blockIdx.z;
    double s = 0.0;
    if (i < g.nx && j < g.ny) {
        const long long c = ((long long)k * g.ny + j) * g.nx + i;
        double rv = 0.0;
        if (c != 0) {
            const long long sy = g.nx, sz = (long long)g.nx * g.ny;
            rv = -rhs[c] - apply7<double>(g, i, j, k, g.wxd, g.wyd, g.wzd, x[c], [&](int a, int b, int d) {
                     return x[c + a + b * sy + d * sz];
                 });
        }
        r[c] = float(rv);
        s = rv * rv;
    }
    const int blk = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    write_partials(partials, blk, &s, 1);
}

// Compatible Neumann form of the pinned system: rows c != 0 unchanged, row 0
// the normal Neumann row with right-hand side -sum_{c != 0} b_c, so every
// row sums to zero. r = b~ - A~ x in FP64, stored in FP32; partial r.r.
__global__ void __launch_bounds__(kBX * kBY) fcg_residual_neumann(Geo3 g, const double *__restrict__ x,
                                                                  const double *__restrict__ rhs,
                                                                  const FcgScalars *sc, float *r, double *partials) {
    const int i = blockIdx.x * kBX + (threadIdx.x & 31), j = blockIdx.y * kBY + (threadIdx.x >> 5), k = blockIdx.z;
    double s = 0.0;
    if (i < g.nx && j < g.ny) {
        const long long c = ((long long)k * g.ny + j) * g.nx + i;
        const long long sy = g.nx, sz = (long long)g.nx * g.ny;
        const double b = c == 0 ? sc->rhs_sum : -rhs[c];
        const double rv = b - apply7<double>(g, i, j, k, g.wxd, g.wyd, g.wzd, x[c], [&](int a, int bb, int d) {
                              return x[c + a + bb * sy + d * sz];
                          });
        r[c] = float(rv);
        s = rv * rv;
    }
    const int blk = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    write_partials(partials, blk, &s, 1);
}

// Partial sums of rhs over the cells other than 0.
__global__ void __launch_bounds__(kPw) fcg_rhs_sum(const double *rhs, long long n, double *partials) {
    __shared__ double red[kPw / 32];
    double s = 0.0;
    for (long long c = blockIdx.x * (long long)kPw + threadIdx.x; c < n; c += (long long)gridDim.x * kPw)
        if (c != 0) s += rhs[c];
    s = block_sum<kPw>(s, red);
    if (threadIdx.x == 0) partials[blockIdx.x * 2] = s;
}

// x -= x_0 (back to the pinned solution, x_0 = 0); x_0 read beforehand.
__global__ void fcg_read_x0(const double *x, FcgScalars *sc) { sc->x0 = x[0]; }
__global__ void __launch_bounds__(kPw) fcg_shift(double *x, const FcgScalars *sc, long long n) {
    const double s = sc->x0;
    for (long long c = blockIdx.x * (long long)kPw + threadIdx.x; c < n; c += (long long)gridDim.x * kPw) x[c] -= s;
}

// Smoothing passes of the preconditioner (damped Jacobi on A~, weight
// omega; pre: z = omega D^-1 r and r - A~ z; post: z_in + omega D^-1
// (r - A~ z_in)) and the operator pass, as z-marching FP32 stencil passes.
// A block owns a 32 x kBY column of cells over kMZ planes; each thread keeps
// the operand of the plane below, its own and the one above in registers,
// so a plane is read from memory once per block (x and y neighbours come
// through L1), and the block's partial sums are reduced once, after the
// march. The operator arithmetic per cell is that of apply7, in its order.
constexpr int kMZ = 16;  // planes per marching block

// omega / diag of the Neumann-form operator by missing-neighbour class
// 9 mx + 3 my + mz (FP32, formed in FP64 on the host), so the smoothing
// passes multiply instead of dividing.
struct SmoothW {
    float winv[27];
};
__device__ __forceinline__ int miss3(int i, int n) { return (i == 0) + (i == n - 1); }
__device__ __forceinline__ float winv_at(const SmoothW &w, const Geo3 &g, int i, int j, int k) {
    return w.winv[9 * miss3(i, g.nx) + 3 * miss3(j, g.ny) + miss3(k, g.nz)];
}

// q = A~ d (Neumann form, FP32); partials d.q and d.r.
__global__ void __launch_bounds__(kBX * kBY) fcg_spmv_m(Geo3 g, const float *__restrict__ d,
                                                        const float *__restrict__ r, float *q, double *partials) {
    const int i = blockIdx.x * kBX + (threadIdx.x & 31), j = blockIdx.y * kBY + (threadIdx.x >> 5);
    const int k0 = blockIdx.z * kMZ, k1 = min(g.nz, k0 + kMZ);
    double v[2] = {0.0, 0.0};
    if (i < g.nx && j < g.ny) {
        const long long sy = g.nx, sz = (long long)g.nx * g.ny;
        long long c = ((long long)k0 * g.ny + j) * g.nx + i;
        float below = k0 > 0 ? d[c - sz] : 0.f, cur = d[c];
        for (int k = k0; k < k1; ++k, c += sz) {
            const float above = k + 1 < g.nz ? d[c + sz] : 0.f;
            const float qv = apply7<float>(g, i, j, k, g.wx, g.wy, g.wz, cur, [&](int a, int b, int e) {
                return e < 0 ? below : (e > 0 ? above : d[c + a + b * sy]);
            });
            q[c] = qv;
            v[0] += double(cur) * double(qv);
            v[1] += double(cur) * double(r[c]);
            below = cur;
            cur = above;
        }
    }
    const int blk = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    write_partials(partials, blk, v, 2);
}

// Pre-smoothing: z_out = omega D^-1 r, r_out = r - A~ z_out.
__global__ void __launch_bounds__(kBX * kBY) fcg_presmooth_m(Geo3 g, const float *__restrict__ r, float *z_out,
                                                             float *r_out, const __grid_constant__ SmoothW w) {
    const int i = blockIdx.x * kBX + (threadIdx.x & 31), j = blockIdx.y * kBY + (threadIdx.x >> 5);
    const int k0 = blockIdx.z * kMZ, k1 = min(g.nz, k0 + kMZ);
    if (i >= g.nx || j >= g.ny) return;
    const long long sy = g.nx, sz = (long long)g.nx * g.ny;
    long long c = ((long long)k0 * g.ny + j) * g.nx + i;
    auto zat = [&](long long m, int ii, int jj, int kk) { return r[m] * winv_at(w, g, ii, jj, kk); };
    float below = k0 > 0 ? zat(c - sz, i, j, k0 - 1) : 0.f, cur = zat(c, i, j, k0);
    for (int k = k0; k < k1; ++k, c += sz) {
        const float above = k + 1 < g.nz ? zat(c + sz, i, j, k + 1) : 0.f;
        const float az = apply7<float>(g, i, j, k, g.wx, g.wy, g.wz, cur, [&](int a, int b, int e) {
            return e < 0 ? below : (e > 0 ? above : zat(c + a + b * sy, i + a, j + b, k));
        });
        z_out[c] = cur;
        r_out[c] = r[c] - az;
        below = cur;
        cur = above;
    }
}

// Post-smoothing of z_in = z_pre + z_net (the coarse correction joins the
// pre-smoothed part on the fly): z_out = z_in + omega D^-1 (r - A~ z_in).
__global__ void __launch_bounds__(kBX * kBY) fcg_postsmooth_m(Geo3 g, const float *__restrict__ r,
                                                              const float *__restrict__ z_pre,
                                                              const float *__restrict__ z_net, float *z_out,
                                                              const __grid_constant__ SmoothW w) {
    const int i = blockIdx.x * kBX + (threadIdx.x & 31), j = blockIdx.y * kBY + (threadIdx.x >> 5);
    const int k0 = blockIdx.z * kMZ, k1 = min(g.nz, k0 + kMZ);
    if (i >= g.nx || j >= g.ny) return;
    const long long sy = g.nx, sz = (long long)g.nx * g.ny;
    long long c = ((long long)k0 * g.ny + j) * g.nx + i;
    auto zin = [&](long long m) { return z_pre[m] + z_net[m]; };
    float below = k0 > 0 ? zin(c - sz) : 0.f, cur = zin(c);
    for (int k = k0; k < k1; ++k, c += sz) {
        const float above = k + 1 < g.nz ? zin(c + sz) : 0.f;
        const float az = apply7<float>(g, i, j, k, g.wx, g.wy, g.wz, cur, [&](int a, int b, int e) {
            return e < 0 ? below : (e > 0 ? above : zin(c + a + b * sy));
        });
        const float res = r[c] - az;
        z_out[c] = cur + res * winv_at(w, g, i, j, k);
        below = cur;
        cur = above;
    }
}

__device__ __forceinline__ void pw_partial(double *partials, double s) {
    __shared__ double red[kPw / 32];
    s = block_sum<kPw>(s, red);
    if (threadIdx.x == 0) partials[blockIdx.x * 2] = s;
}

// x += alpha d (FP64), r -= alpha q (FP32); partial r.r.
__global__ void __launch_bounds__(kPw) fcg_update(double *x, float *r, const float *d, const float *q,
                                                  const FcgScalars *sc, long long n4, double *partials) {
    const double alpha = sc->alpha;
    const float af = float(alpha);
    double s = 0.0;
    for (long long t = blockIdx.x * (long long)kPw + threadIdx.x; t < n4; t += (long long)gridDim.x * kPw) {
        const float4 dv = reinterpret_cast<const float4 *>(d)[t];
        const float4 qv = reinterpret_cast<const float4 *>(q)[t];
        float4 rv = reinterpret_cast<float4 *>(r)[t];
        double2 *x2 = reinterpret_cast<double2 *>(x) + 2 * t;
        double2 xa = x2[0], xb = x2[1];
        xa.x += alpha * dv.x; xa.y += alpha * dv.y; xb.x += alpha * dv.z; xb.y += alpha * dv.w;
        x2[0] = xa;
        x2[1] = xb;
        rv.x -= af * qv.x; rv.y -= af * qv.y; rv.z -= af * qv.z; rv.w -= af * qv.w;
        reinterpret_cast<float4 *>(r)[t] = rv;
        s += double(rv.x) * rv.x + double(rv.y) * rv.y + double(rv.z) * rv.z + double(rv.w) * rv.w;
    }
    pw_partial(partials, s);
}

// Partials z . q_j (j < count) and sum z, kDotStride per block.
__global__ void __launch_bounds__(kPw) fcg_dots(const float *z, DirSet ds, long long n4, double *partials) {
    __shared__ double red[kPw / 32];
    double s[kMaxM + 1];
    #pragma unroll
    for (int j = 0; j <= kMaxM; ++j) s[j] = 0.0;
    for (long long t = blockIdx.x * (long long)kPw + threadIdx.x; t < n4; t += (long long)gridDim.x * kPw) {
        const float4 u = reinterpret_cast<const float4 *>(z)[t];
        s[kMaxM] += double(u.x) + double(u.y) + double(u.z) + double(u.w);
        #pragma unroll
        for (int j = 0; j < kMaxM; ++j) {
            if (j >= ds.count) break;
            const float4 v = reinterpret_cast<const float4 *>(ds.q[j])[t];
            s[j] += double(u.x) * v.x + double(u.y) * v.y + double(u.z) * v.z + double(u.w) * v.w;
        }
    }
    for (int j = 0; j <= kMaxM; ++j) {
        if (j < kMaxM && j >= ds.count) continue;  // uniform over the block
        const double t = block_sum<kPw>(s[j], red);
        if (threadIdx.x == 0) partials[(long long)blockIdx.x * kDotStride + j] = t;
    }
}

// d = (z - mean z) - sum_j coef_j d_j: A~-orthogonal to the stored
// directions and orthogonal to the constants (the null space of A~).
__global__ void __launch_bounds__(kPw) fcg_direction(const float *z, float *d, DirSet ds, const FcgScalars *sc,
                                                     long long n4) {
    const float m = float(sc->zmean);
    float c[kMaxM];
    #pragma unroll
    for (int j = 0; j < kMaxM; ++j) c[j] = j < ds.count ? float(sc->coef[j]) : 0.f;
    for (long long t = blockIdx.x * (long long)kPw + threadIdx.x; t < n4; t += (long long)gridDim.x * kPw) {
        const float4 zv = reinterpret_cast<const float4 *>(z)[t];
        float4 dv = make_float4(zv.x - m, zv.y - m, zv.z - m, zv.w - m);
        #pragma unroll
        for (int j = 0; j < kMaxM; ++j) {
            if (j >= ds.count) break;
            const float4 o = reinterpret_cast<const float4 *>(ds.d[j])[t];
            dv.x -= c[j] * o.x; dv.y -= c[j] * o.y; dv.z -= c[j] * o.z; dv.w -= c[j] * o.w;
        }
        reinterpret_cast<float4 *>(d)[t] = dv;
    }
}

enum FinalizeMode { kFinRR = 0, kFinSpmv = 1, kFinRhsSum = 3 };

// Fixed-order reduction of the partials (stride 2) into the scalars of one
// step; kFinSpmv also stores d.q in ring slot `slot`.
__global__ void __launch_bounds__(1024) fcg_finalize(const double *partials, int np, int mode, FcgScalars *sc,
                                                     int slot) {
    __shared__ double red[32];
    const bool two = mode == kFinSpmv;
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) {
        a += partials[2 * i];
        if (two) b += partials[2 * i + 1];
    }
    a = block_sum<1024>(a, red);
    if (two) b = block_sum<1024>(b, red);
    if (threadIdx.x != 0) return;
    if (mode == kFinRR) {
        sc->rr = a;
    } else if (mode == kFinRhsSum) {
        sc->rhs_sum = a;
    } else {
        sc->dq = a;
        sc->dr = b;
        sc->dqs[slot] = a;
        const bool bad = !(a > 1e-300) || !isfinite(a) || !isfinite(b);
        sc->breakdown = bad ? 1 : 0;
        sc->alpha = bad ? 0.0 : b / a;
    }
}

// coef_j = (z . q_j) / (d_j . q_j) and mean z from the fcg_dots partials.
// (z - mean z) . q_j = z . q_j because q_j = A~ d_j sums to zero.
__global__ void __launch_bounds__(1024) fcg_finalize_dots(const double *partials, int np, DirSet ds, FcgScalars *sc,
                                                          double inv_n) {
    __shared__ double red[32];
    for (int j = 0; j <= kMaxM; ++j) {
        if (j < kMaxM && j >= ds.count) continue;
        double a = 0.0;
        for (int i = threadIdx.x; i < np; i += blockDim.x) a += partials[(long long)i * kDotStride + j];
        a = block_sum<1024>(a, red);
        if (threadIdx.x == 0) {
            if (j == kMaxM) {
                sc->zmean = a * inv_n;
            } else {
                const double c = a / sc->dqs[ds.slot[j]];
                sc->coef[j] = c;
                if (!isfinite(c)) sc->breakdown = 1;
            }
        }
    }
}

int pw_grid(long long n4) { return (int)std::max<long long>(1, std::min<long long>((n4 + kPw - 1) / kPw, kMaxPwBlocks)); }

}  // namespace

// Device buffers of one FCG solve.
struct FcgWork {
    int nx = 0, ny = 0, nz = 0;
    float *r = nullptr, *z = nullptr;
    float *t1 = nullptr, *t2 = nullptr;  // smoothed residual and coarse correction
    float *dd[kMaxM] = {}, *qq[kMaxM] = {};  // stored directions and their A~ images
    int ndirs = 0;
    cudaError_t ensure_dirs(int m) {
        const long long n = (long long)nx * ny * nz;
        for (; ndirs < m; ++ndirs) {
            cudaError_t e = cudaMalloc(&dd[ndirs], 4 * n);
            if (e == cudaSuccess) e = cudaMalloc(&qq[ndirs], 4 * n);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    double *partials = nullptr;
    FcgScalars *sc = nullptr, *h_sc = nullptr;
    // two event pairs around the network (an application can be queued
    // ahead of the one being read) and the event of the scalar read-back
    cudaEvent_t e0[2] = {nullptr, nullptr}, e1[2] = {nullptr, nullptr}, esc = nullptr;
    cudaError_t ensure(int nx_, int ny_, int nz_) {
        if (r && nx_ == nx && ny_ == ny && nz_ == nz) return cudaSuccess;
        release();
        const long long n = (long long)nx_ * ny_ * nz_;
        const long long np = std::max<long long>((long long)((nx_ + kBX - 1) / kBX) * ((ny_ + kBY - 1) / kBY) * nz_,
                                                 kMaxPwBlocks);
        cudaError_t e = cudaMalloc(&r, 4 * n);
        if (e == cudaSuccess) e = cudaMalloc(&z, 4 * n);
        if (e == cudaSuccess) e = cudaMalloc(&t1, 4 * n);
        if (e == cudaSuccess) e = cudaMalloc(&t2, 4 * n);
        if (e == cudaSuccess) e = cudaMalloc(&partials, sizeof(double) * std::max<long long>(2 * np, kDotStride * kMaxPwBlocks));
        if (e == cudaSuccess) e = cudaMalloc(&sc, sizeof(FcgScalars));
        if (e == cudaSuccess) e = cudaMallocHost(&h_sc, sizeof(FcgScalars));
        for (int k = 0; k < 2; ++k) {
            if (e == cudaSuccess) e = cudaEventCreate(&e0[k]);
            if (e == cudaSuccess) e = cudaEventCreate(&e1[k]);
        }
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&esc, cudaEventDisableTiming);
        if (e == cudaSuccess) { nx = nx_; ny = ny_; nz = nz_; }
        return e;
    }
    void release() {
        cudaFree(r); cudaFree(z); cudaFree(t1); cudaFree(t2); cudaFree(partials);
        cudaFree(sc);
        for (int j = 0; j < ndirs; ++j) {
            cudaFree(dd[j]);
            cudaFree(qq[j]);
            dd[j] = qq[j] = nullptr;
        }
        ndirs = 0;
        if (h_sc) cudaFreeHost(h_sc);
        for (int k = 0; k < 2; ++k) {
            if (e0[k]) cudaEventDestroy(e0[k]);
            if (e1[k]) cudaEventDestroy(e1[k]);
            e0[k] = e1[k] = nullptr;
        }
        if (esc) cudaEventDestroy(esc);
        esc = nullptr;
        r = z = t1 = t2 = nullptr;
        partials = nullptr;
        sc = h_sc = nullptr;
        nx = ny = nz = 0;
    }
};

}  // namespace flursys

// The network behind FlursysFcgNet: BF16 copies, the FP32 master parameters
// it was built from, and its workspace.
struct FlursysFcgNet {
    int device = 0;
    flursys::NetWeights w;
    float *master = nullptr;  // FP32 parameters (device)
    flursys::NetWorkspace ws;
    flursys::FcgWork fcg;
    flursys::PcgWorkspace pcg;  // fallback Jacobi-PCG (allocated on first use)
    int pcg_nx = 0, pcg_ny = 0, pcg_nz = 0;
    std::string err;
};

namespace flursys {

namespace {

int32_t net_fail(std::string *dst, const std::string &msg, int32_t code) {
    *dst = msg;
    return code;
}

}  // namespace

int32_t fcg_solve(FlursysFcgNet *net, int nx, int ny, int nz, double dx, double dy, double dz, double *x,
                  const double *rhs, double atol, double rtol, long long max_iters, int precision_fallback,
                  cudaStream_t st, FlursysFcgReport *rep, std::string *err) {
    FcgWork &f = net->fcg;
    std::memset(rep, 0, sizeof *rep);
    if (nx % 8 || ny % 8 || nz % 8)
        return net_fail(err, "the learned FCG needs nx, ny and nz divisible by 8", FLURSYS_ERR_UNSUPPORTED);
    cudaError_t e = f.ensure(nx, ny, nz);
    if (e != cudaSuccess) return set_cuda_error(err, e, "FCG workspace");
    Geo3 g{nx, ny, nz, 0.f, 0.f, 0.f, 1.0 / (dx * dx), 1.0 / (dy * dy), 1.0 / (dz * dz)};
    g.wx = float(g.wxd); g.wy = float(g.wyd); g.wz = float(g.wzd);
    const double h2 = 3.0 / (g.wxd + g.wyd + g.wzd);
    const long long n = (long long)nx * ny * nz, n4 = n / 4;
    const dim3 sgrid((nx + kBX - 1) / kBX, (ny + kBY - 1) / kBY, nz), sblock(kBX * kBY);
    const int nsb = (int)(sgrid.x * sgrid.y * sgrid.z), npw = pw_grid(n4);
    const dim3 mgrid(sgrid.x, sgrid.y, (nz + kMZ - 1) / kMZ);  // z-marching passes
    const int nmb = (int)(mgrid.x * mgrid.y * mgrid.z);
    double net_ms = 0.0;
    auto sync_scalars = [&]() -> cudaError_t {
        cudaError_t m = cudaMemcpyAsync(f.h_sc, f.sc, sizeof(FcgScalars), cudaMemcpyDeviceToHost, st);
        if (m == cudaSuccess) m = cudaStreamSynchronize(st);
        return m;
    };
    const double inv_n = 1.0 / double(n);
    auto residual = [&]() -> cudaError_t {  // pinned system (the stop rule's r0 and the final check)
        fcg_residual<<<sgrid, sblock, 0, st>>>(g, x, rhs, f.r, f.partials);
        fcg_finalize<<<1, 1024, 0, st>>>(f.partials, nsb, kFinRR, f.sc, 0);
        return cudaGetLastError();
    };
    auto residual_neumann = [&]() -> cudaError_t {  // the iterated compatible Neumann form
        fcg_residual_neumann<<<sgrid, sblock, 0, st>>>(g, x, rhs, f.sc, f.r, f.partials);
        fcg_finalize<<<1, 1024, 0, st>>>(f.partials, nsb, kFinRR, f.sc, 0);
        return cudaGetLastError();
    };
    auto shift = [&]() -> cudaError_t {  // x -= x_0: the pinned solution
        fcg_read_x0<<<1, 1, 0, st>>>(x, f.sc);
        fcg_shift<<<npw, kPw, 0, st>>>(x, f.sc, n);
        return cudaGetLastError();
    };
    // M(r): damped-Jacobi pre-smoothing, the network on the smoothed residual,
    // damped-Jacobi post-smoothing (smooth = 0: the network alone).
    const char *smooth_env = std::getenv("FLURSYS_FCG_SMOOTH");
    const bool smooth = !(smooth_env && smooth_env[0] == '0');
    // damped-Jacobi weight of the smoothers (FLURSYS_FCG_OMEGA, 0 < omega < 2)
    const char *omega_env = std::getenv("FLURSYS_FCG_OMEGA");
    const double omega_set = omega_env ? std::atof(omega_env) : 0.8;
    const double omega = omega_set > 0.0 && omega_set < 2.0 ? omega_set : 0.8;
    SmoothW sw{};
    for (int t = 0; t < 27; ++t) {
        const int mx = t / 9, my = (t / 3) % 3, mz = t % 3;
        const double dg = (2 - mx) * g.wxd + (2 - my) * g.wyd + (2 - mz) * g.wzd;
        sw.winv[t] = dg > 0.0 ? float(omega / dg) : 0.f;
    }
    // pair: the event pair timing this application of the network
    auto precondition = [&](int pair) -> cudaError_t {
        cudaError_t m = cudaSuccess;
        if (!smooth) {
            cudaEventRecord(f.e0[pair], st);
            m = net_apply(net->w, net->ws, nx, ny, nz, h2, f.r, f.z, st);
            cudaEventRecord(f.e1[pair], st);
            return m;
        }
        fcg_presmooth_m<<<mgrid, sblock, 0, st>>>(g, f.r, f.t2, f.t1, sw);  // t2 = z0, t1 = r - A z0
        cudaEventRecord(f.e0[pair], st);
        m = net_apply(net->w, net->ws, nx, ny, nz, h2, f.t1, f.z, st);   // z = N(r1)
        cudaEventRecord(f.e1[pair], st);
        if (m != cudaSuccess) return m;
        fcg_postsmooth_m<<<mgrid, sblock, 0, st>>>(g, f.r, f.t2, f.z, f.t1, sw);  // t1 = post-smoothed z0 + N(r1)
        std::swap(f.z, f.t1);                                                      // z = the preconditioned residual
        return cudaGetLastError();
    };
    e = residual();
    if (e == cudaSuccess) e = sync_scalars();
    if (e != cudaSuccess) return set_cuda_error(err, e, "FCG initial residual");
    const double r0 = std::sqrt(f.h_sc->rr);
    const double threshold = atol + rtol * r0;
    rep->initial_residual = r0;
    // The iteration runs on the compatible Neumann form, whose residual
    // bounds the pinned one once x is shifted to x_0 = 0.
    fcg_rhs_sum<<<npw, kPw, 0, st>>>(rhs, n, f.partials);
    fcg_finalize<<<1, 1024, 0, st>>>(f.partials, npw, kFinRhsSum, f.sc, 0);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = residual_neumann();
    if (e == cudaSuccess) e = sync_scalars();
    if (e != cudaSuccess) return set_cuda_error(err, e, "FCG initial residual");
    double res = std::sqrt(f.h_sc->rr);
    long long its = 0;
    bool converged = r0 <= threshold, fallback = false;
    double window_res = res;
    // residual at the last replacement (or the start): the FP32 recurrence
    // is replaced by the FP64 true residual once it has fallen 1000-fold
    // below it, so the rounding the recurrence accumulated while the
    // residual was large never exceeds ~1e-4 of the current residual
    // (reliable updates, after van der Vorst and Ye)
    double rep_ref = res;
    // stored directions (1..8): 8 by default (measured at 256^3 on B200 with
    // the shipped network: 67-70 iterations and 121.6 ms per warm-started
    // solve for m = 8, 69-74 and 124.9 ms for m = 6, 76-84 for m = 4)
    const char *m_env = std::getenv("FLURSYS_FCG_M");
    const int mdirs = m_env ? std::max(1, std::min(kMaxM, std::atoi(m_env))) : kDefaultM;
    e = f.ensure_dirs(mdirs);
    if (e != cudaSuccess) return set_cuda_error(err, e, "FCG direction storage");
    const char *trace_env = std::getenv("FLURSYS_FCG_TRACE");  // per-iteration scalars to stderr
    const bool trace = trace_env && trace_env[0] == '1';
    // The host reads each iteration's scalars while the GPU already runs the
    // next iteration's preconditioner M(r), which only reads r and writes the
    // scratch vectors: it is kept when the iteration goes on unchanged and
    // recomputed after a residual replacement (which rewrites r); a
    // replacement due by the iteration count is not speculated on.
    int pair = 0;            // event pair of the application this iteration uses
    bool pre_ready = false;  // M(r) of this iteration was queued at the end of the previous one
    for (long long it = 0; !converged && !fallback; ++it) {
        if (it >= max_iters) { fallback = true; break; }
        // z = M(r); d = z - sum_j coef_j d_j over the last m directions
        e = pre_ready ? cudaSuccess : precondition(pair);
        pre_ready = false;
        DirSet ds{};
        ds.count = (int)std::min<long long>(it, mdirs);
        for (int j = 0; j < ds.count; ++j) {
            const int sl = (int)((it - 1 - j) % mdirs);
            ds.slot[j] = sl;
            ds.d[j] = f.dd[sl];
            ds.q[j] = f.qq[sl];
        }
        const int slot = (int)(it % mdirs);
        float *dcur = f.dd[slot], *qcur = f.qq[slot];
        if (e == cudaSuccess) {
            fcg_dots<<<npw, kPw, 0, st>>>(f.z, ds, n4, f.partials);
            fcg_finalize_dots<<<1, 1024, 0, st>>>(f.partials, npw, ds, f.sc, inv_n);
            fcg_direction<<<npw, kPw, 0, st>>>(f.z, dcur, ds, f.sc, n4);
            fcg_spmv_m<<<mgrid, sblock, 0, st>>>(g, dcur, f.r, qcur, f.partials);
            fcg_finalize<<<1, 1024, 0, st>>>(f.partials, nmb, kFinSpmv, f.sc, slot);
            fcg_update<<<npw, kPw, 0, st>>>(x, f.r, dcur, qcur, f.sc, n4, f.partials);
            fcg_finalize<<<1, 1024, 0, st>>>(f.partials, npw, kFinRR, f.sc, 0);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(f.h_sc, f.sc, sizeof(FcgScalars), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaEventRecord(f.esc, st);
        // (not when the last residual read was within 3x of the threshold:
        // the solve is about to stop and the queued application would be lost)
        const bool speculate = e == cudaSuccess && (it + 1) % 50 != 0 && it + 1 < max_iters && res > 3.0 * threshold;
        if (speculate) e = precondition(1 - pair);
        if (e == cudaSuccess) e = cudaEventSynchronize(f.esc);
        if (e != cudaSuccess) return set_cuda_error(err, e, "FCG iteration");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, f.e0[pair], f.e1[pair]);
        net_ms += ms;
        its = it + 1;
        if (trace)
            std::fprintf(stderr, "fcg it %lld: |r| %.6e alpha %.6e d.q %.6e d.r %.6e coef0 %.6e\n", its,
                         std::sqrt(f.h_sc->rr), f.h_sc->alpha, f.h_sc->dq, f.h_sc->dr, f.h_sc->coef[0]);
        if (f.h_sc->breakdown) { fallback = true; break; }
        res = std::sqrt(f.h_sc->rr);
        if (!std::isfinite(res)) { fallback = true; break; }
        bool replaced = false;
        if (res <= threshold || its % 50 == 0 || res < 1.0e-3 * rep_ref) {  // FP64 true residual replaces r
            replaced = true;
            e = residual_neumann();
            if (e == cudaSuccess) e = sync_scalars();
            if (e != cudaSuccess) return set_cuda_error(err, e, "FCG residual replacement");
            res = std::sqrt(f.h_sc->rr);
            rep_ref = res;
            if (res <= threshold) { converged = true; break; }
        }
        if (its % 25 == 0) {
            if (res > 0.5 * window_res) { fallback = true; break; }
            window_res = res;
        }
        if (speculate && !replaced) {  // no replacement rewrote r: keep the queued M(r)
            pre_ready = true;
            pair = 1 - pair;
        }
    }
    rep->fcg_iterations = its;
    rep->net_ms = net_ms;
    e = shift();
    if (e != cudaSuccess) return set_cuda_error(err, e, "FCG shift");
    if (!converged) {
        // plain Jacobi-PCG from the current x, same absolute threshold
        if (net->pcg_nx != nx || net->pcg_ny != ny || net->pcg_nz != nz) {
            net->pcg.free_all();
            net->pcg = PcgWorkspace();
            e = net->pcg.allocate3d(nx, ny, nz, precision_fallback, net->device, st);
            if (e != cudaSuccess) return set_cuda_error(err, e, "fallback PCG workspace");
            net->pcg_nx = nx; net->pcg_ny = ny; net->pcg_nz = nz;
        }
        const int32_t s = run_pcg3d(net->pcg, nx, ny, nz, dx, dy, dz, x, rhs, precision_fallback, FLURSYS_STOP_REL_L2,
                                    0.0, threshold, 0.0, std::max<long long>(max_iters, 1) * 100, 50, st, err);
        if (s) return s;
        e = cudaMemcpyAsync(net->pcg.h_result, net->pcg.result, sizeof(PcgResultDev), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return set_cuda_error(err, e, "fallback PCG");
        const int32_t ps = pcg_result_status(*net->pcg.h_result, err);
        if (ps) return ps;
        rep->fallback = 1;
        rep->pcg_iterations = net->pcg.h_result->iterations;
    }
    // final FP64 check
    e = residual();
    if (e == cudaSuccess) e = sync_scalars();
    if (e != cudaSuccess) return set_cuda_error(err, e, "FCG final residual");
    rep->final_residual = std::sqrt(f.h_sc->rr);
    rep->relative_residual = r0 > 0.0 ? rep->final_residual / r0 : 0.0;
    rep->status = rep->final_residual <= threshold ? FLURSYS_LINEAR_CONVERGED : FLURSYS_LINEAR_MAX_ITERATIONS;
    return FLURSYS_OK;
}

// Weights file: "FLNT", uint32 version 1, uint32 layer count, (cin, cout)
// int32 pairs, int64 parameter count, FP32 parameters (little endian).
int32_t fcgnet_read_file(const char *path, std::vector<float> *out, std::string *err) {
    FILE *fp = std::fopen(path, "rb");
    if (!fp) return net_fail(err, std::string("cannot open FCG weights file ") + path, FLURSYS_ERR_INVALID_ARGUMENT);
    char magic[4];
    uint32_t version = 0, layers = 0;
    bool ok = std::fread(magic, 1, 4, fp) == 4 && std::memcmp(magic, "FLNT", 4) == 0 &&
              std::fread(&version, 4, 1, fp) == 1 && version == 1 && std::fread(&layers, 4, 1, fp) == 1 &&
              layers == (uint32_t)kNetLayers;
    for (int l = 0; ok && l < kNetLayers; ++l) {
        int32_t io[2];
        ok = std::fread(io, 4, 2, fp) == 2 && io[0] == kNetCin[l] && io[1] == kNetCout[l];
    }
    int64_t count = 0;
    ok = ok && std::fread(&count, 8, 1, fp) == 1 && count == net_param_count();
    if (ok) {
        out->resize(count);
        ok = std::fread(out->data(), 4, count, fp) == (size_t)count;
    }
    std::fclose(fp);
    if (!ok) return net_fail(err, std::string("FCG weights file does not match the network: ") + path,
                             FLURSYS_ERR_INVALID_ARGUMENT);
    for (float v : *out)
        if (!std::isfinite(v)) return net_fail(err, "FCG weights file holds non-finite values", FLURSYS_ERR_NON_FINITE);
    return FLURSYS_OK;
}

int32_t fcgnet_create(const float *host_params, FlursysFcgNet **out, std::string *err) {
    auto *net = new FlursysFcgNet();
    cudaGetDevice(&net->device);
    cudaError_t e = net->w.allocate();
    if (e == cudaSuccess) e = cudaMalloc(&net->master, sizeof(float) * net_param_count());
    if (e == cudaSuccess) {
        if (host_params)
            e = cudaMemcpy(net->master, host_params, sizeof(float) * net_param_count(), cudaMemcpyHostToDevice);
        else
            e = cudaMemset(net->master, 0, sizeof(float) * net_param_count());
    }
    if (e == cudaSuccess) e = net_pack_weights(net->master, net->w, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        fcgnet_destroy(net);
        return set_cuda_error(err, e, "creating the FCG network");
    }
    *out = net;
    return FLURSYS_OK;
}

void fcgnet_destroy(FlursysFcgNet *net) {
    if (!net) return;
    net->w.release();
    net->ws.release();
    net->fcg.release();
    net->pcg.free_all();
    if (net->master) cudaFree(net->master);
    delete net;
}

}  // namespace flursys

using namespace flursys;

extern "C" int64_t flursys_cuda_fcgnet_param_count(void) { return net_param_count(); }

extern "C" int32_t flursys_cuda_fcgnet_create(const float *params, FlursysFcgNet **out) {
    if (!out) return FLURSYS_ERR_INVALID_ARGUMENT;
    std::string err;
    const int32_t s = fcgnet_create(params, out, &err);
    if (s) set_global_error(err);
    return s;
}

extern "C" int32_t flursys_cuda_fcgnet_load(const char *path, FlursysFcgNet **out) {
    if (!path || !out) return FLURSYS_ERR_INVALID_ARGUMENT;
    std::vector<float> p;
    std::string err;
    int32_t s = fcgnet_read_file(path, &p, &err);
    if (!s) s = fcgnet_create(p.data(), out, &err);
    if (s) set_global_error(err);
    return s;
}

extern "C" int32_t flursys_cuda_fcgnet_set_params(FlursysFcgNet *net, const float *params_device, void *stream) {
    if (!net || !params_device) return FLURSYS_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(net->master, params_device, sizeof(float) * net_param_count(),
                                    cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = net_pack_weights(net->master, net->w, st);
    if (e != cudaSuccess) {
        set_global_error(std::string("fcgnet_set_params: ") + cudaGetErrorString(e));
        return FLURSYS_ERR_CUDA;
    }
    return FLURSYS_OK;
}

extern "C" int32_t flursys_cuda_fcgnet_get_params(const FlursysFcgNet *net, float *host, int64_t count) {
    if (!net || !host || count != net_param_count()) return FLURSYS_ERR_INVALID_ARGUMENT;
    const cudaError_t e = cudaMemcpy(host, net->master, sizeof(float) * count, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        set_global_error(std::string("fcgnet_get_params: ") + cudaGetErrorString(e));
        return FLURSYS_ERR_CUDA;
    }
    return FLURSYS_OK;
}

extern "C" int32_t flursys_cuda_fcgnet_apply(FlursysFcgNet *net, int64_t nx, int64_t ny, int64_t nz, double h2,
                                             const float *r_device, float *z_device, void *stream) {
    if (!net || !r_device || !z_device || nx < 8 || ny < 8 || nz < 8 || nx % 8 || ny % 8 || nz % 8 ||
        nx * ny * nz >= (1LL << 31)) {
        set_global_error("fcgnet_apply: need device buffers and nx, ny, nz >= 8, divisible by 8");
        return FLURSYS_ERR_INVALID_ARGUMENT;
    }
    const cudaError_t e = net_apply(net->w, net->ws, (int)nx, (int)ny, (int)nz, h2, r_device, z_device,
                                    static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        set_global_error(std::string("fcgnet_apply: ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? FLURSYS_ERR_OUT_OF_MEMORY : FLURSYS_ERR_CUDA;
    }
    return FLURSYS_OK;
}

extern "C" int32_t flursys_cuda_fcgnet_train_sample(FlursysFcgNet *net, int64_t nx, int64_t ny, int64_t nz,
                                                    const float *b_hat, const float *p_hat, double norm,
                                                    int32_t loss_kind, float *grad_device, double *loss_device,
                                                    void *stream) {
    if (!net || !b_hat || !p_hat || !grad_device || !loss_device || !(norm > 0.0) || nx < 8 || ny < 8 || nz < 8 ||
        nx % 8 || ny % 8 || nz % 8 || nx * ny * nz >= (1LL << 31) ||
        (loss_kind != FLURSYS_FCG_LOSS_ENERGY && loss_kind != FLURSYS_FCG_LOSS_RESIDUAL)) {
        set_global_error("fcgnet_train_sample: need device buffers, norm > 0, a known loss and nx, ny, nz >= 8, "
                         "divisible by 8");
        return FLURSYS_ERR_INVALID_ARGUMENT;
    }
    const cudaError_t e = net_train_sample(net->w, net->ws, (int)nx, (int)ny, (int)nz, b_hat, p_hat, norm, loss_kind,
                                           grad_device, loss_device, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        set_global_error(std::string("fcgnet_train_sample: ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? FLURSYS_ERR_OUT_OF_MEMORY : FLURSYS_ERR_CUDA;
    }
    return FLURSYS_OK;
}

extern "C" int32_t flursys_cuda_fcgnet_adam(float *w, const float *g, float *m, float *v, int64_t n, float lr,
                                            float beta1, float beta2, float eps, int64_t t, float grad_scale,
                                            void *stream) {
    if (!w || !g || !m || !v || n < 1 || t < 1) return FLURSYS_ERR_INVALID_ARGUMENT;
    const cudaError_t e = net_adam(w, g, m, v, n, lr, beta1, beta2, eps, t, grad_scale, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        set_global_error(std::string("fcgnet_adam: ") + cudaGetErrorString(e));
        return FLURSYS_ERR_CUDA;
    }
    return FLURSYS_OK;
}

extern "C" int32_t flursys_cuda_fcgnet_destroy(FlursysFcgNet *net) {
    fcgnet_destroy(net);
    return FLURSYS_OK;
}

extern "C" int32_t flursys_cuda_stencil_fcg(FlursysFcgNet *net, int64_t nx, int64_t ny, int64_t nz, double dx,
                                            double dy, double dz, const double *rhs, double *x_inout,
                                            const FlursysLinearSolverOptions *options, FlursysFcgReport *report) {
    if (!net || !rhs || !x_inout || !options || !report || nx < 8 || ny < 8 || nz < 8 ||
        nx * ny * nz >= (1LL << 31)) {
        set_global_error("stencil_fcg: null argument or grid below 8^3 or above 2^31 cells");
        return FLURSYS_ERR_INVALID_ARGUMENT;
    }
    if (!(std::isfinite(options->absolute_tolerance) && options->absolute_tolerance >= 0.0 &&
          std::isfinite(options->relative_tolerance) && options->relative_tolerance >= 0.0)) {
        set_global_error("iterative solver breakdown: invalid solver tolerance");
        return FLURSYS_ERR_BREAKDOWN;
    }
    const long long n = nx * ny * nz;
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return FLURSYS_ERR_CUDA;
    double *dxp = nullptr, *drhs = nullptr;
    std::string err;
    int32_t status = FLURSYS_OK;
    cudaError_t e = cudaMalloc(&dxp, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&drhs, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dxp, x_inout, sizeof(double) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(drhs, rhs, sizeof(double) * n, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) status = set_cuda_error(&err, e, "stencil FCG setup");
    if (!status)
        status = fcg_solve(net, (int)nx, (int)ny, (int)nz, dx, dy, dz, dxp, drhs, options->absolute_tolerance,
                           options->relative_tolerance, options->max_iterations, FLURSYS_PRECISION_MIXED, st, report,
                           &err);
    if (!status) {
        e = cudaMemcpyAsync(x_inout, dxp, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) status = set_cuda_error(&err, e, "stencil FCG");
    }
    cudaFree(dxp);
    cudaFree(drhs);
    cudaStreamDestroy(st);
    if (status) set_global_error(err);
    return status;
}
