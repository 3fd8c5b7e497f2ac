// pcg3d_res.cu — the 3D pressure PCG (MIXED) with its FP32 state held on the
// chip for the whole solve.
//
// When every tile of 32 x 32 x tz cells (tz <= 16) gets an SM of its own, one
// cooperative launch runs the complete solve: each block keeps its tile's
// search direction d (with a one-cell face halo), q = A d and the FP32
// solution increment in shared memory and the residual r in registers, so an
// iteration touches HBM or L2 only for the residual's tile faces (the halo
// exchange) and for the per-block partial sums. Two grid barriers per
// iteration carry the two PCG reductions (d.q; r.r, r.z, max|r|); the faces
// of r are published before the second one, and after it every block forms
// d = z + beta d on its halo from its neighbours' faces and its own copy of
// the old halo, with the owners' arithmetic, so halo and owner values are
// bit-identical.
//
// The system, iteration order, precisions and stop semantics are those of
// the graph-driven PCG (pcg3d_seq.cu), after the reference's PCG order
// (src/solver/incompressible.rs:1125-1186) on the pinned 7-point system of
// src/solver/incompressible_3d.rs:293-332: FP32 stencil and vectors, FP64
// dot products and scalars, the FP32 increment folded into the FP64
// pressure and r replaced by the FP64 b - A x every `replace_every`
// iterations and before convergence is accepted, then the FP64 ||b - A x||_2
// of the returned pressure. Every block computes every reduction in the
// same fixed order, so all blocks take the same decisions.
//
// Two forms share the tile layout. The two-reduction form above serves
// every stop rule. For the L2 stop rule the single-reduction form
// (pcg3d_res1_kernel) needs one grid barrier per iteration: the halo keeps
// its own copy of r (in the registers of the threads that own the halo
// cells), the faces of q = A d are exchanged instead of those of r, and one
// reduction carries (r,r), (r,z), (d,q), (q,q), (q,Mq), (q,r), (q,z) and
// max|r| of the same iteration. alpha = (r,z)/(d,q) uses the directly summed
// (r,z); the (r,z) and ||r||^2 of the next residual r - alpha q come from
// the exact expansions (r,z) - 2 alpha (q,z) + alpha^2 (q,Mq) and
// (r,r) - 2 alpha (q,r) + alpha^2 (q,q) of the summed products, so beta and
// the stop test are decided where the reference's PCG decides them, and the
// next reduction sums (r,z) directly again (no recurrence accumulates). The
// vector updates are FP32 fused multiply-adds with alpha rounded to FP32,
// the same alpha for the increment and the residual (so the two stay
// consistent); dots and scalars stay FP64, each product formed from the
// FP32 factors widened once per cell.
//
// Every grid-barrier wait is bounded; a barrier that gives up sets the
// timeout bit in CgSeqState::device_error and the blocks return.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "common.cuh"
#include "pcg3d_res.cuh"

namespace flursys {

namespace {

constexpr int RX = 32, RY = 32;
constexpr int kResBlock = 512;            // threads; each owns columns (tx, ty) and (tx, ty + 16)
constexpr int kCols = RX * RY / kResBlock;  // columns per thread
constexpr int kResMaxTz = 16;
constexpr int HX = RX + 2, HY = RY + 2;
constexpr int kResSlots = 8;  // partial sums per block and reduction (7 sums and a maximum at most)
constexpr int kResMaxBlocks = 160;                    // one block per SM
constexpr int kResPerLane = (kResMaxBlocks + 31) / 32;  // partials per lane in a grid reduction
// face values per thread: two 32 x 32 z-faces and four 32 x tz side faces
constexpr int kHaloPer = (2 * RX * RY + 4 * RX * kResMaxTz + kResBlock - 1) / kResBlock;

__device__ __forceinline__ int rmiss(int i, int n) { return (i == 0) + (i == n - 1); }

size_t res_smem_bytes(int tz) {
    return sizeof(float) * ((size_t)HX * HY * (tz + 2) + 2 * (size_t)RX * RY * tz);
}

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid barrier of the resident solve: one arrival ticket per block on a
// counter that only grows (cleared before each launch); barrier number t
// is complete when the counter reaches (t + 1) * nblocks, so the arrival
// is a single atomic and the wait polls the same word. The wait is
// bounded; a failure sets the timeout bit in the barrier's error word and
// in the state, and every block leaves at its next barrier.
__device__ __forceinline__ bool res_sync(const ResArgs &a, unsigned long long *wait_ns = nullptr) {
    const unsigned nblocks = gridDim.x + (unsigned)a.barrier_extra;
    __syncthreads();
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        const unsigned long long tw = wait_ns ? gtimer() : 0ull;
        unsigned *cnt = &a.bar->count;
        unsigned old;
        asm volatile("atom.add.release.gpu.u32 %0, [%1], 1;" : "=r"(old) : "l"(cnt) : "memory");
        const unsigned target = (old / nblocks + 1u) * nblocks;
        int ok = 1;
        long long spins = 0;
        for (;;) {
            unsigned cur;
            asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(cur) : "l"(cnt) : "memory");
            if ((int)(cur - target) >= 0) break;
            if ((++spins & 63) == 0) {
                const unsigned err = *(volatile unsigned *)&a.bar->error;
                if (err != 0u || spins > a.spin_limit) {
                    atomicOr(&a.bar->error, (unsigned)kDevErrBarrierTimeout);
                    atomicOr(&a.st->device_error, (unsigned)kDevErrBarrierTimeout);
                    ok = 0;
                    break;
                }
            }
        }
        asm volatile("fence.acq_rel.gpu;" ::: "memory");
        if (wait_ns) *wait_ns += gtimer() - tw;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

struct ResCtx {
    const ResArgs &a;
    float *dsm, *dxs, *qs;
    double *red;
    int round;
    unsigned long long t_reduce;  // thread 0: time in grid reductions
    unsigned long long t_wait;    // thread 0: time waiting inside their grid barriers
};

// Sums NS values (and, with MAX, the maximum of one more) over the grid.
// Every block obtains the same bits. Returns false when the barrier failed.
template <int BLK, int NS, bool MAX>
__device__ __forceinline__ bool grid_reduce(ResCtx &c, double (&v)[NS], double &mx) {
    static_assert(NS + (MAX ? 1 : 0) <= kResSlots && NS + (MAX ? 1 : 0) <= BLK / 32, "reduction width");
    const unsigned long long t0 = gtimer();
    block_reduce_n<BLK, NS, MAX>(v, mx, c.red);
    const int nb = gridDim.x;
    double *P = c.a.partials + (size_t)(c.round & 1) * nb * kResSlots;
    ++c.round;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NS; ++k) P[blockIdx.x * kResSlots + k] = v[k];
        if (MAX) P[blockIdx.x * kResSlots + NS] = mx;
    }
    if (!res_sync(c.a, &c.t_wait)) return false;
    // warp k sums value k over the blocks (every block in the same order)
    const int wk = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (wk < NS + (MAX ? 1 : 0)) {
        const bool is_max = MAX && wk == NS;
        // every partial this lane needs is requested before the first is used
        double p[kResPerLane];
#pragma unroll
        for (int u = 0; u < kResPerLane; ++u) {
            const int b = lane + 32 * u;
            p[u] = b < nb ? __ldcg(P + b * kResSlots + wk) : 0.0;
        }
        double t = 0.0;
#pragma unroll
        for (int u = 0; u < kResPerLane; ++u) t = is_max ? fmax(t, p[u]) : t + p[u];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double p = __shfl_xor_sync(0xffffffffu, t, o);
            t = is_max ? fmax(t, p) : t + p;
        }
        if (lane == 0) c.red[wk] = t;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NS; ++k) v[k] = c.red[k];
    if (MAX) mx = c.red[NS];
    __syncthreads();
    c.t_reduce += gtimer() - t0;
    return true;
}

// d = z + beta d_old with z = r / diag in FP32 (the pinned cell stays 0).
__device__ __forceinline__ float make_d(float r, float dold, float idg, bool pin, bool first, float beta) {
    if (pin) return 0.f;
    const float z = __fmul_rn(r, idg);
    return first ? z : __fmaf_rn(beta, dold, z);
}

__global__ void __launch_bounds__(kResBlock, 1) pcg3d_res2_kernel(const __grid_constant__ ResArgs a) {
    extern __shared__ float smem[];
    __shared__ double red[8 * (kResBlock / 32)];
    __shared__ float idgf[27];
    const int tz_full = a.tz;
    float *dsm = smem;                                      // (tz + 2) x HY x HX
    float *dxs = smem + (size_t)HX * HY * (tz_full + 2);   // tz x RY x RX
    float *qs = dxs + (size_t)RX * RY * tz_full;           // tz x RY x RX
    ResCtx c{a, dsm, dxs, qs, red, 0, 0ull, 0ull};
    unsigned long long t_halo = 0, t_op = 0, t_upd = 0;
    const int b = blockIdx.x;
    const int i0 = (b % a.ntx) * RX, j0 = ((b / a.ntx) % a.nty) * RY, k0 = (b / (a.ntx * a.nty)) * a.tz;
    const int kz = min(a.tz, a.nz - k0);
    const int tx = threadIdx.x & 31;
    // Per owned column h: y offset in the tile, validity, neighbour weights.
    int ty[kCols], col[kCols], cls_xy[kCols];
    bool in[kCols], pcol[kCols], face_col[kCols];
    float wxy[kCols][4];   // x-, x+, y-, y+ (FP32)
    double dxy[kCols][4];  // the same in FP64
#pragma unroll
    for (int h = 0; h < kCols; ++h) {
        ty[h] = (threadIdx.x >> 5) + h * (kResBlock / 32);
        const int i = i0 + tx, j = j0 + ty[h];
        in[h] = i < a.nx && j < a.ny;
        col[h] = in[h] ? j * a.nx + i : 0;
        pcol[h] = in[h] && col[h] == 0;
        face_col[h] = tx == 0 || tx == RX - 1 || ty[h] == 0 || ty[h] == RY - 1;
        cls_xy[h] = in[h] ? 9 * rmiss(i, a.nx) + 3 * rmiss(j, a.ny) : 0;
        const bool w = in[h] && i > 0, e = in[h] && i + 1 < a.nx, s = in[h] && j > 0, n = in[h] && j + 1 < a.ny;
        wxy[h][0] = w ? a.wx : 0.f; wxy[h][1] = e ? a.wx : 0.f;
        wxy[h][2] = s ? a.wy : 0.f; wxy[h][3] = n ? a.wy : 0.f;
        dxy[h][0] = w ? a.ix2 : 0.0; dxy[h][1] = e ? a.ix2 : 0.0;
        dxy[h][2] = s ? a.iy2 : 0.0; dxy[h][3] = n ? a.iy2 : 0.0;
    }
    auto own = [&](int h, int kk) { return ((kk + 1) * HY + ty[h] + 1) * HX + tx + 1; };  // dsm slot
    auto loc = [&](int h, int kk) { return (kk * RY + ty[h]) * RX + tx; };               // dxs / qs slot

    if (threadIdx.x < 27) idgf[threadIdx.x] = a.inv_diag_f[threadIdx.x];
    for (int s = threadIdx.x; s < HX * HY * (tz_full + 2); s += kResBlock) dsm[s] = 0.f;
    for (int s = threadIdx.x; s < RX * RY * tz_full; s += kResBlock) dxs[s] = 0.f;
    __syncthreads();

    float r[kCols][kResMaxTz];
#pragma unroll
    for (int h = 0; h < kCols; ++h)
#pragma unroll
        for (int kk = 0; kk < kResMaxTz; ++kk) r[h][kk] = 0.f;

    // r = b - A x in FP64 (b = -rhs), rounded to FP32; sums of the rounded r.
    // With `final_pass` only the FP64 sum of (b - A x)^2 is formed.
    auto residual = [&](double &srr, double &srz, double &smax, bool final_pass) {
#pragma unroll
        for (int h = 0; h < kCols; ++h) {
            if (!in[h]) continue;
#pragma unroll
            for (int kk = 0; kk < kResMaxTz; ++kk) {
                if (kk >= kz) continue;
                const int k = k0 + kk;
                const int cc = col[h] + k * a.nxy;
                const bool pin = pcol[h] && k == 0;
                auto xv = [&](int idx) -> double { return idx == 0 ? 0.0 : __ldcg(a.x + idx); };
                const double cur = pin ? 0.0 : __ldcg(a.x + cc);
                const double wzm = k > 0 ? a.iz2 : 0.0, wzp = k + 1 < a.nz ? a.iz2 : 0.0;
                const double *w = dxy[h];
                const double xm = w[0] != 0.0 ? xv(cc - 1) : 0.0, xp = w[1] != 0.0 ? xv(cc + 1) : 0.0;
                const double ym = w[2] != 0.0 ? xv(cc - a.nx) : 0.0, yp = w[3] != 0.0 ? xv(cc + a.nx) : 0.0;
                const double zm = k > 0 ? xv(cc - a.nxy) : 0.0, zp = k + 1 < a.nz ? xv(cc + a.nxy) : 0.0;
                const double ax = (w[0] + w[1] + w[2] + w[3] + wzm + wzp) * cur -
                                  (w[0] * xm + w[1] * xp + w[2] * ym + w[3] * yp + wzm * zm + wzp * zp);
                const double t = pin ? 0.0 : -__ldg(a.rhs + cc) - ax;
                if (final_pass) {
                    srr += t * t;
                    continue;
                }
                const float rv = float(t);
                r[h][kk] = rv;
                const double rd = double(rv);
                srr += rd * rd;
                srz += rd * rd * (pin ? 1.0 : a.inv_diag[cls_xy[h] + rmiss(k, a.nz)]);
                smax = fmax(smax, fabs(rd));
            }
        }
    };
    // Publishes the residual of the tile's face cells for the neighbours' halos.
    auto publish = [&]() {
#pragma unroll
        for (int h = 0; h < kCols; ++h) {
            if (!in[h]) continue;
#pragma unroll
            for (int kk = 0; kk < kResMaxTz; ++kk) {
                if (kk >= kz) continue;
                if (face_col[h] || kk == 0 || kk == kz - 1) a.face0[col[h] + (k0 + kk) * a.nxy] = r[h][kk];
            }
        }
    };
    // x += dx on the tile (FP64 pressure; the pinned cell stays 0), dx = 0.
    auto fold = [&]() {
#pragma unroll
        for (int h = 0; h < kCols; ++h) {
            if (!in[h]) continue;
            for (int kk = 0; kk < kz; ++kk) {
                const int cc = col[h] + (k0 + kk) * a.nxy;
                if (cc == 0) a.x[0] = 0.0;
                else a.x[cc] += double(dxs[loc(h, kk)]);
                dxs[loc(h, kk)] = 0.f;
            }
        }
    };

    // ---- initial residual ----
    if (b == 0 && threadIdx.x == 0) a.x[0] = 0.0;
    if (!res_sync(a)) return;
    double sums[2] = {0.0, 0.0};
    double smax = 0.0;
    residual(sums[0], sums[1], smax, false);
    publish();
    if (!grid_reduce<kResBlock, 2, true>(c, sums, smax)) return;
    const bool l2 = a.stop_rule == FLURSYS_STOP_REL_L2;
    auto stop_ok = [&](double res, double thr) { return l2 ? res <= thr : res < thr; };
    const double initial_l2 = sqrt(sums[0]);
    const double initial = l2 ? initial_l2 : smax;
    const double threshold = l2 ? a.atol + a.rtol * initial : a.tol;
    double residual_v = initial, rz_old = sums[1], beta = 0.0;
    bool first = true;
    long long iterations = 0;
    int status = stop_ok(initial, threshold) ? FLURSYS_LINEAR_CONVERGED : FLURSYS_LINEAR_MAX_ITERATIONS;
    int error = 0;
    bool done = status == FLURSYS_LINEAR_CONVERGED || a.max_iters <= 0;

    const int nhalo = 2 * RX * RY + 4 * RX * kz;
    while (!done) {
        // ---- d = z + beta d_old on the halo (neighbours' r faces) and the tile ----
        const unsigned long long t0 = gtimer();
        const float fb = float(beta);
        // every face value this thread needs is requested before any is used
        float hv[kHaloPer];
        int hslot[kHaloPer], hcls[kHaloPer];
#pragma unroll
        for (int u = 0; u < kHaloPer; ++u) {
            const int s = threadIdx.x + u * kResBlock;
            hslot[u] = -1;
            hv[u] = 0.f;
            hcls[u] = 0;
            if (s >= nhalo) continue;
            int xx, yy, kk;
            if (s < 2 * RX * RY) {
                const int t = s & (RX * RY - 1);
                xx = t & 31; yy = t >> 5; kk = s < RX * RY ? -1 : kz;
            } else {
                const int t = s - 2 * RX * RY, f = t / (RX * kz), w = t - f * (RX * kz);
                const int p = w & 31, q = w >> 5;
                if (f < 2) { xx = p; yy = f == 0 ? -1 : RY; kk = q; }
                else { yy = p; xx = f == 2 ? -1 : RX; kk = q; }
            }
            const int gi = i0 + xx, gj = j0 + yy, gk = k0 + kk;
            if (gi < 0 || gi >= a.nx || gj < 0 || gj >= a.ny || gk < 0 || gk >= a.nz) continue;
            const int cc = (gk * a.ny + gj) * a.nx + gi;
            hslot[u] = ((kk + 1) * HY + yy + 1) * HX + xx + 1;
            hcls[u] = cc == 0 ? -1 : 9 * rmiss(gi, a.nx) + 3 * rmiss(gj, a.ny) + rmiss(gk, a.nz);
            hv[u] = __ldcg(a.face0 + cc);
        }
#pragma unroll
        for (int u = 0; u < kHaloPer; ++u) {
            if (hslot[u] < 0) continue;
            const int sl = hslot[u];
            dsm[sl] = make_d(hv[u], dsm[sl], idgf[hcls[u] < 0 ? 0 : hcls[u]], hcls[u] < 0, first, fb);
        }
#pragma unroll
        for (int h = 0; h < kCols; ++h) {
            if (!in[h]) continue;
#pragma unroll
            for (int kk = 0; kk < kResMaxTz; ++kk) {
                if (kk >= kz) continue;
                const int k = k0 + kk;
                const int sl = own(h, kk);
                dsm[sl] = make_d(r[h][kk], dsm[sl], idgf[cls_xy[h] + rmiss(k, a.nz)], pcol[h] && k == 0, first, fb);
            }
        }
        __syncthreads();
        const unsigned long long t1 = gtimer();
        t_halo += t1 - t0;
        // ---- q = A d on the tile, d.q ----
        double sdq[1] = {0.0};
#pragma unroll
        for (int h = 0; h < kCols; ++h) {
            if (!in[h]) continue;
            const float *w = wxy[h];
            float below = dsm[own(h, -1)], cur = dsm[own(h, 0)];
            for (int kk = 0; kk < kz; ++kk) {
                const int k = k0 + kk;
                const int sp = own(h, kk);
                const float above = dsm[sp + HX * HY];
                const float wzm = k > 0 ? a.wz : 0.f, wzp = k + 1 < a.nz ? a.wz : 0.f;
                float ax = (w[0] + w[1] + w[2] + w[3] + wzm + wzp) * cur -
                           (w[0] * dsm[sp - 1] + w[1] * dsm[sp + 1] + w[2] * dsm[sp - HX] + w[3] * dsm[sp + HX] +
                            wzm * below + wzp * above);
                if (pcol[h] && k == 0) ax = cur;  // identity row of the pinned cell
                qs[loc(h, kk)] = ax;
                sdq[0] += double(cur) * double(ax);
                below = cur;
                cur = above;
            }
        }
        double unused = 0.0;
        t_op += gtimer() - t1;
        if (!grid_reduce<kResBlock, 1, false>(c, sdq, unused)) return;
        const unsigned long long t2 = gtimer();
        const double dq = sdq[0];
        if (fabs(dq) < 1.0e-30 || !isfinite(dq) || !isfinite(rz_old / dq)) {
            error = FLURSYS_ERR_BREAKDOWN;
            break;
        }
        const double alpha = rz_old / dq;
        // ---- dx += alpha d, r -= alpha q, sums ----
        double s2[2] = {0.0, 0.0};
        double mx = 0.0;
#pragma unroll
        for (int h = 0; h < kCols; ++h) {
            if (!in[h]) continue;
#pragma unroll
            for (int kk = 0; kk < kResMaxTz; ++kk) {
                if (kk >= kz) continue;
                const int k = k0 + kk;
                const int l = loc(h, kk);
                dxs[l] = float(double(dxs[l]) + alpha * double(dsm[own(h, kk)]));
                r[h][kk] = float(double(r[h][kk]) - alpha * double(qs[l]));
                const double rd = double(r[h][kk]);
                s2[0] += rd * rd;
                s2[1] += rd * rd * ((pcol[h] && k == 0) ? 1.0 : a.inv_diag[cls_xy[h] + rmiss(k, a.nz)]);
                mx = fmax(mx, fabs(rd));
            }
        }
        publish();
        t_upd += gtimer() - t2;
        if (!grid_reduce<kResBlock, 2, true>(c, s2, mx)) return;
        iterations += 1;
        double res = l2 ? sqrt(s2[0]) : mx;
        residual_v = res;
        if (!isfinite(res)) {
            error = FLURSYS_ERR_NON_FINITE;
            break;
        }
        bool conv = stop_ok(res, threshold);
        double rz = s2[1];
        if (conv || (iterations % a.replace_every) == 0) {
            // ---- FP64 residual replacement ----
            const unsigned long long t3 = gtimer();
            fold();
            if (!res_sync(a)) return;
            double s3[2] = {0.0, 0.0};
            double m3 = 0.0;
            residual(s3[0], s3[1], m3, false);
            publish();
            if (!grid_reduce<kResBlock, 2, true>(c, s3, m3)) return;
            res = l2 ? sqrt(s3[0]) : m3;
            residual_v = res;
            if (!isfinite(res)) {
                error = FLURSYS_ERR_NON_FINITE;
                break;
            }
            conv = stop_ok(res, threshold);
            rz = s3[1];
            t_upd += gtimer() - t3;
        }
        if (conv) {
            status = FLURSYS_LINEAR_CONVERGED;
            break;
        }
        if (fabs(rz_old) < 1.0e-30 || iterations >= a.max_iters) break;
        beta = rz / rz_old;
        rz_old = rz;
        first = false;
    }
    // ---- fold a pending increment, then the FP64 ||b - A x||_2 ----
    if (status != FLURSYS_LINEAR_CONVERGED) fold();
    if (!res_sync(a)) return;
    double st[1] = {0.0};
    double d0 = 0.0, d1 = 0.0;
    residual(st[0], d0, d1, true);
    double unused = 0.0;
    if (!grid_reduce<kResBlock, 1, false>(c, st, unused)) return;
    if (b == 0 && threadIdx.x == 0) {
        CgSeqState *w = a.st;
        w->error = error;
        w->status = status;
        w->iterations = iterations;
        w->initial = initial;
        w->initial_l2 = initial_l2;
        w->residual = residual_v;
        w->threshold = threshold;
        w->true_l2 = sqrt(st[0]);
        w->done = 1;
        w->phase_ns[0] = t_halo;
        w->phase_ns[1] = t_op;
        w->phase_ns[2] = c.t_reduce;
        w->phase_ns[3] = t_upd;
    }
}


// Single-reduction form for the L2 stop rule (see the file comment).
template <int BLK, bool COL32>
__global__ void __launch_bounds__(BLK, 1) pcg3d_res1_kernel(const __grid_constant__ ResArgs a) {
    constexpr int kC = RX * RY / BLK;                                       // columns per thread
    constexpr int kHP = (2 * RX * RY + 4 * RX * kResMaxTz + BLK - 1) / BLK;  // halo cells per thread
    extern __shared__ float smem[];
    __shared__ double red[8 * (BLK / 32)];
    __shared__ float idgf[27];
    const int tz_full = a.tz;
    float *dsm = smem;                                      // (tz + 2) x HY x HX
    float *dxs = smem + (size_t)HX * HY * (tz_full + 2);   // tz x RY x RX
    float *qs = dxs + (size_t)RX * RY * tz_full;           // tz x RY x RX
    ResCtx c{a, dsm, dxs, qs, red, 0, 0ull, 0ull};
    unsigned long long t_halo = 0, t_op = 0, t_upd = 0;
    const int b = blockIdx.x;
    const int i0 = (b % a.ntx) * RX, j0 = ((b / a.ntx) % a.nty) * RY, k0 = (b / (a.ntx * a.nty)) * a.tz;
    const int kz = min(a.tz, a.nz - k0);
    const int tx = threadIdx.x & 31;
    int ty[kC], col[kC], cls_xy[kC];
    bool in[kC], pcol[kC], face_col[kC];
    float wxy[kC][4];  // x-, x+, y-, y+ operator weights (0 at a wall)
#pragma unroll
    for (int h = 0; h < kC; ++h) {
        ty[h] = (threadIdx.x >> 5) + h * (BLK / 32);
        const int i = i0 + tx, j = j0 + ty[h];
        in[h] = i < a.nx && j < a.ny;
        col[h] = in[h] ? j * a.nx + i : 0;
        pcol[h] = in[h] && col[h] == 0;
        face_col[h] = tx == 0 || tx == RX - 1 || ty[h] == 0 || ty[h] == RY - 1;
        cls_xy[h] = in[h] ? 9 * rmiss(i, a.nx) + 3 * rmiss(j, a.ny) : 0;
        wxy[h][0] = in[h] && i > 0 ? a.wx : 0.f;
        wxy[h][1] = in[h] && i + 1 < a.nx ? a.wx : 0.f;
        wxy[h][2] = in[h] && j > 0 ? a.wy : 0.f;
        wxy[h][3] = in[h] && j + 1 < a.ny ? a.wy : 0.f;
    }
    auto own = [&](int h, int kk) { return ((kk + 1) * HY + ty[h] + 1) * HX + tx + 1; };
    auto loc = [&](int h, int kk) { return (kk * RY + ty[h]) * RX + tx; };

    // The halo cells this thread keeps: shared-memory slot | class << 16
    // (class 27: the pinned cell), global index; -1 when none.
    int hpk[kHP], hcc[kHP];
    const int nhalo = 2 * RX * RY + 4 * RX * kz;
#pragma unroll
    for (int u = 0; u < kHP; ++u) {
        const int s = threadIdx.x + u * BLK;
        hpk[u] = -1;
        hcc[u] = 0;
        if (s >= nhalo) continue;
        int xx, yy, kk;
        if (s < 2 * RX * RY) {
            const int t = s & (RX * RY - 1);
            xx = t & 31; yy = t >> 5; kk = s < RX * RY ? -1 : kz;
        } else {
            const int t = s - 2 * RX * RY, f = t / (RX * kz), w = t - f * (RX * kz);
            const int p = w & 31, q = w >> 5;
            if (f < 2) { xx = p; yy = f == 0 ? -1 : RY; kk = q; }
            else { yy = p; xx = f == 2 ? -1 : RX; kk = q; }
        }
        const int gi = i0 + xx, gj = j0 + yy, gk = k0 + kk;
        if (gi < 0 || gi >= a.nx || gj < 0 || gj >= a.ny || gk < 0 || gk >= a.nz) continue;
        const int cc = (gk * a.ny + gj) * a.nx + gi;
        const int cls = cc == 0 ? 27 : 9 * rmiss(gi, a.nx) + 3 * rmiss(gj, a.ny) + rmiss(gk, a.nz);
        hpk[u] = (((kk + 1) * HY + yy + 1) * HX + xx + 1) | (cls << 16);
        hcc[u] = cc;
    }

    if (threadIdx.x < 27) idgf[threadIdx.x] = a.inv_diag_f[threadIdx.x];
    for (int s = threadIdx.x; s < HX * HY * (tz_full + 2); s += BLK) dsm[s] = 0.f;
    for (int s = threadIdx.x; s < RX * RY * tz_full; s += BLK) dxs[s] = 0.f;
    __syncthreads();

    float r[kC][kResMaxTz];
    float hr[kHP];
#pragma unroll
    for (int h = 0; h < kC; ++h)
#pragma unroll
        for (int kk = 0; kk < kResMaxTz; ++kk) r[h][kk] = 0.f;
#pragma unroll
    for (int u = 0; u < kHP; ++u) hr[u] = 0.f;
    int fr = 0;  // face exchanges so far; exchange f uses buffer f & 1
    auto face = [&](int f) { return (f & 1) ? a.face1 : a.face0; };

    // r = b - A x in FP64 (b = -rhs) on the tile, rounded to FP32, with the
    // sums of the rounded r; with `final_pass` only the FP64 sum of (b - A x)^2.
    auto residual = [&](double &srr, double &srz, double &smax, bool final_pass) {
#pragma unroll
        for (int h = 0; h < kC; ++h) {
            if (!in[h]) continue;
            const double wxm = wxy[h][0] != 0.f ? a.ix2 : 0.0, wxp = wxy[h][1] != 0.f ? a.ix2 : 0.0;
            const double wym = wxy[h][2] != 0.f ? a.iy2 : 0.0, wyp = wxy[h][3] != 0.f ? a.iy2 : 0.0;
#pragma unroll
            for (int kk = 0; kk < kResMaxTz; ++kk) {
                if (kk >= kz) continue;
                const int k = k0 + kk;
                const int cc = col[h] + k * a.nxy;
                const bool pin = pcol[h] && k == 0;
                auto xv = [&](int idx) -> double { return idx == 0 ? 0.0 : __ldcg(a.x + idx); };
                const double cur = pin ? 0.0 : __ldcg(a.x + cc);
                const double wzm = k > 0 ? a.iz2 : 0.0, wzp = k + 1 < a.nz ? a.iz2 : 0.0;
                const double xm = wxm != 0.0 ? xv(cc - 1) : 0.0, xp = wxp != 0.0 ? xv(cc + 1) : 0.0;
                const double ym = wym != 0.0 ? xv(cc - a.nx) : 0.0, yp = wyp != 0.0 ? xv(cc + a.nx) : 0.0;
                const double zm = k > 0 ? xv(cc - a.nxy) : 0.0, zp = k + 1 < a.nz ? xv(cc + a.nxy) : 0.0;
                const double ax = (wxm + wxp + wym + wyp + wzm + wzp) * cur -
                                  (wxm * xm + wxp * xp + wym * ym + wyp * yp + wzm * zm + wzp * zp);
                const double t = pin ? 0.0 : -__ldg(a.rhs + cc) - ax;
                if (final_pass) {
                    srr += t * t;
                    continue;
                }
                const float rv = float(t);
                r[h][kk] = rv;
                const double rd = double(rv);
                srr += rd * rd;
                srz += rd * rd * (pin ? 1.0 : a.inv_diag[cls_xy[h] + rmiss(k, a.nz)]);
                smax = fmax(smax, fabs(rd));
            }
        }
    };
    // The tile's face values of r, then (after the next grid barrier) the
    // halo's r from the neighbours' faces.
    auto publish_r = [&](float *fb) {
#pragma unroll
        for (int h = 0; h < kC; ++h) {
            if (!in[h]) continue;
#pragma unroll
            for (int kk = 0; kk < kResMaxTz; ++kk) {
                if (kk >= kz) continue;
                if (face_col[h] || kk == 0 || kk == kz - 1) fb[col[h] + (k0 + kk) * a.nxy] = r[h][kk];
            }
        }
    };
    auto fetch_halo_r = [&](const float *fb) {
#pragma unroll
        for (int u = 0; u < kHP; ++u)
            if (hpk[u] >= 0) hr[u] = __ldcg(fb + hcc[u]);
    };
    auto fold = [&]() {
#pragma unroll
        for (int h = 0; h < kC; ++h) {
            if (!in[h]) continue;
            for (int kk = 0; kk < kz; ++kk) {
                const int cc = col[h] + (k0 + kk) * a.nxy;
                if (cc == 0) a.x[0] = 0.0;
                else a.x[cc] += double(dxs[loc(h, kk)]);
                dxs[loc(h, kk)] = 0.f;
            }
        }
    };

    // ---- initial residual and its halo ----
    if (b == 0 && threadIdx.x == 0) a.x[0] = 0.0;
    if (!res_sync(a)) return;
    double s0[2] = {0.0, 0.0};
    double m0 = 0.0;
    residual(s0[0], s0[1], m0, false);
    publish_r(face(fr));
    if (!grid_reduce<BLK, 2, true>(c, s0, m0)) return;
    fetch_halo_r(face(fr));
    ++fr;
    const double initial_l2 = sqrt(s0[0]);
    const double initial = initial_l2;
    const double threshold = a.atol + a.rtol * initial;
    double residual_v = initial, beta = 0.0;
    bool first = true;
    long long iterations = 0;
    int status = initial <= threshold ? FLURSYS_LINEAR_CONVERGED : FLURSYS_LINEAR_MAX_ITERATIONS;
    int error = 0;
    bool done = status == FLURSYS_LINEAR_CONVERGED || a.max_iters <= 0;

    while (!done) {
        // ---- d = z + beta d_old on the tile and its halo ----
        const unsigned long long t0 = gtimer();
        const float fb = float(beta);
#pragma unroll
        for (int u = 0; u < kHP; ++u) {
            if (hpk[u] < 0) continue;
            const int sl = hpk[u] & 0xffff, cls = hpk[u] >> 16;
            dsm[sl] = make_d(hr[u], dsm[sl], idgf[cls == 27 ? 0 : cls], cls == 27, first, fb);
        }
#pragma unroll
        for (int h = 0; h < kC; ++h) {
            if (!in[h]) continue;
#pragma unroll
            for (int kk = 0; kk < kResMaxTz; ++kk) {
                if (kk >= kz) continue;
                const int k = k0 + kk;
                const int sl = own(h, kk);
                dsm[sl] = make_d(r[h][kk], dsm[sl], idgf[cls_xy[h] + rmiss(k, a.nz)], pcol[h] && k == 0, first, fb);
            }
        }
        __syncthreads();
        const unsigned long long t1 = gtimer();
        t_halo += t1 - t0;
        // ---- q = A d on the tile, q's faces out, and the sums ----
        // S: (r,r), (r,z), (d,q), (q,q), (q,Mq), (q,r), (q,z)
        double S[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        float rmax = 0.f;
        float *fq = face(fr);
        const bool zlo = k0 == 0, zhi = k0 + kz == a.nz;  // the tile holds the plane k = 0 / k = nz - 1
#pragma unroll
        for (int h = 0; h < kC; ++h) {
            if (!in[h]) continue;
            const float *w = wxy[h];
            // Jacobi weights: the column's class inside, its z-wall class at k = 0, nz - 1
            const double wm = a.inv_diag[cls_xy[h]], we = a.inv_diag[cls_xy[h] + 1] - wm;
            // the column's sums: FP32 over its tz cells (COL32) or FP64 per cell
            double crr = 0.0, cqq = 0.0, cqr = 0.0, cdq = 0.0;
            float frr = 0.f, fqq = 0.f, fqr = 0.f, fdq = 0.f;
            float below = dsm[own(h, -1)], cur = dsm[own(h, 0)];
#pragma unroll
            for (int kk = 0; kk < kResMaxTz; ++kk) {
                if (kk >= kz) continue;
                const int k = k0 + kk;
                const int sp = own(h, kk);
                const float above = dsm[sp + HX * HY];
                const float wzm = k > 0 ? a.wz : 0.f, wzp = k + 1 < a.nz ? a.wz : 0.f;
                float ax = (w[0] + w[1] + w[2] + w[3] + wzm + wzp) * cur -
                           (w[0] * dsm[sp - 1] + w[1] * dsm[sp + 1] + w[2] * dsm[sp - HX] + w[3] * dsm[sp + HX] +
                            wzm * below + wzp * above);
                if (pcol[h] && k == 0) ax = cur;  // identity row of the pinned cell
                qs[loc(h, kk)] = ax;
                if (face_col[h] || kk == 0 || kk == kz - 1) fq[col[h] + k * a.nxy] = ax;
                if (COL32) {
                    const float rv = r[h][kk];
                    frr = __fmaf_rn(rv, rv, frr);
                    fqq = __fmaf_rn(ax, ax, fqq);
                    fqr = __fmaf_rn(ax, rv, fqr);
                    fdq = __fmaf_rn(cur, ax, fdq);
                } else {
                    const double rd = double(r[h][kk]), qd = double(ax), dd = double(cur);
                    crr = fma(rd, rd, crr);
                    cqq = fma(qd, qd, cqq);
                    cqr = fma(qd, rd, cqr);
                    cdq = fma(dd, qd, cdq);
                }
                if ((kk == 0 && zlo) || (kk == kz - 1 && zhi)) {  // a z-wall cell: its class weight
                    const double rd = double(r[h][kk]), qd = double(ax);
                    S[1] = fma(we, rd * rd, S[1]);
                    S[4] = fma(we, qd * qd, S[4]);
                    S[6] = fma(we, qd * rd, S[6]);
                }
                rmax = fmaxf(rmax, fabsf(r[h][kk]));
                below = cur;
                cur = above;
            }
            if (COL32) {
                crr = double(frr); cqq = double(fqq); cqr = double(fqr); cdq = double(fdq);
            }
            S[0] += crr;
            S[1] = fma(wm, crr, S[1]);
            S[2] += cdq;
            S[3] += cqq;
            S[4] = fma(wm, cqq, S[4]);
            S[5] += cqr;
            S[6] = fma(wm, cqr, S[6]);
        }
        double mx = double(rmax);
        const unsigned long long t2 = gtimer();
        t_op += t2 - t1;
        if (!grid_reduce<BLK, 7, true>(c, S, mx)) return;
        const unsigned long long t3 = gtimer();
        const double rz = S[1], dq = S[2];
        if (fabs(dq) < 1.0e-30 || !isfinite(dq) || !isfinite(rz / dq)) {
            error = FLURSYS_ERR_BREAKDOWN;
            break;
        }
        const double alpha = rz / dq;
        const double rr_next = S[0] - 2.0 * alpha * S[5] + alpha * alpha * S[3];
        double rz_next = S[1] - 2.0 * alpha * S[6] + alpha * alpha * S[4];
        // ---- dx += alpha d, r -= alpha q on the tile and the halo ----
        const float af = float(alpha);
        const float *fqr = face(fr);
        ++fr;
        float hq[kHP];
#pragma unroll
        for (int u = 0; u < kHP; ++u) hq[u] = hpk[u] >= 0 ? __ldcg(fqr + hcc[u]) : 0.f;
#pragma unroll
        for (int h = 0; h < kC; ++h) {
            if (!in[h]) continue;
#pragma unroll
            for (int kk = 0; kk < kResMaxTz; ++kk) {
                if (kk >= kz) continue;
                const int l = loc(h, kk);
                dxs[l] = __fmaf_rn(af, dsm[own(h, kk)], dxs[l]);
                r[h][kk] = __fmaf_rn(-af, qs[l], r[h][kk]);
            }
        }
#pragma unroll
        for (int u = 0; u < kHP; ++u) hr[u] = __fmaf_rn(-af, hq[u], hr[u]);
        iterations += 1;
        double res = sqrt(fmax(rr_next, 0.0));
        residual_v = res;
        if (!isfinite(res)) {
            error = FLURSYS_ERR_NON_FINITE;
            break;
        }
        bool conv = res <= threshold;
        if (conv || (iterations % a.replace_every) == 0) {
            // ---- FP64 residual replacement ----
            fold();
            if (!res_sync(a)) return;
            double s3[2] = {0.0, 0.0};
            double m3 = 0.0;
            residual(s3[0], s3[1], m3, false);
            publish_r(face(fr));
            if (!grid_reduce<BLK, 2, true>(c, s3, m3)) return;
            fetch_halo_r(face(fr));
            ++fr;
            res = sqrt(s3[0]);
            residual_v = res;
            if (!isfinite(res)) {
                error = FLURSYS_ERR_NON_FINITE;
                break;
            }
            conv = res <= threshold;
            rz_next = s3[1];
        }
        t_upd += gtimer() - t3;
        if (conv) {
            status = FLURSYS_LINEAR_CONVERGED;
            break;
        }
        if (fabs(rz) < 1.0e-30 || iterations >= a.max_iters) break;
        beta = rz_next / rz;
        first = false;
    }
    // ---- fold a pending increment, then the FP64 ||b - A x||_2 ----
    if (status != FLURSYS_LINEAR_CONVERGED) fold();
    if (!res_sync(a)) return;
    double st[1] = {0.0};
    double d0 = 0.0, d1 = 0.0;
    residual(st[0], d0, d1, true);
    double unused = 0.0;
    if (!grid_reduce<BLK, 1, false>(c, st, unused)) return;
    if (b == 0 && threadIdx.x == 0) {
        CgSeqState *w = a.st;
        w->error = error;
        w->status = status;
        w->iterations = iterations;
        w->initial = initial;
        w->initial_l2 = initial_l2;
        w->residual = residual_v;
        w->threshold = threshold;
        w->true_l2 = sqrt(st[0]);
        w->done = 1;
        w->phase_ns[0] = t_halo;
        w->phase_ns[1] = t_op;
        w->phase_ns[2] = c.t_reduce;
        w->phase_ns[3] = t_upd;
        w->phase_ns[4] = c.t_wait;
    }
    if (threadIdx.x == 0) atomicMax(&a.st->phase_ns[5], t_halo + t_op + t_upd);
}

}  // namespace

bool pcg3d_res_plan(Pcg3dResPlan &plan, const Pcg3dArgs &args, int device) {
    plan = Pcg3dResPlan{};
    const char *env = std::getenv("FLURSYS_PCG_RESIDENT");
    if (env && std::strcmp(env, "0") == 0) return false;
    if (args.nz < 2) return false;
    ResArgs &a = plan.args;
    a.nx = args.nx; a.ny = args.ny; a.nz = args.nz;
    a.nxy = args.nx * args.ny;
    a.n = a.nxy * args.nz;
    a.ntx = (a.nx + RX - 1) / RX;
    a.nty = (a.ny + RY - 1) / RY;
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return false;
    const long long cols = (long long)a.ntx * a.nty;
    if (cols > sms) return false;
    const int slabs = (int)(sms / cols);
    a.tz = (a.nz + slabs - 1) / slabs;
    if (a.tz > kResMaxTz) return false;
    a.ntz = (a.nz + a.tz - 1) / a.tz;
    plan.grid = (int)(cols * a.ntz);
    if (plan.grid > kResMaxBlocks) return false;
    plan.smem = res_smem_bytes(a.tz);
    // one reduction per iteration for the L2 stop rule (FLURSYS_PCG_RESIDENT=2
    // keeps the two-reduction form)
    plan.single = args.stop_rule == FLURSYS_STOP_REL_L2 && !(env && std::strcmp(env, "2") == 0);
    // every product of the dot products in FP64 (default: the CG inner
    // products are FP64 throughout) or each column's products summed in FP32
    // first (FLURSYS_PCG_RES_DOTS=32)
    const char *denv = std::getenv("FLURSYS_PCG_RES_DOTS");
    plan.col32 = denv && std::atoi(denv) == 32;
    plan.block = kResBlock;
    plan.kernel = !plan.single ? (const void *)pcg3d_res2_kernel
                  : plan.col32 ? (const void *)pcg3d_res1_kernel<kResBlock, true>
                               : (const void *)pcg3d_res1_kernel<kResBlock, false>;
    if (cudaFuncSetAttribute(plan.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plan.smem) != cudaSuccess)
        return false;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, plan.kernel, plan.block, plan.smem) != cudaSuccess ||
        per_sm < 1 || plan.grid > per_sm * sms)
        return false;
    a.ix2 = args.ix2; a.iy2 = args.iy2; a.iz2 = args.iz2;
    a.wx = float(args.ix2); a.wy = float(args.iy2); a.wz = float(args.iz2);
    for (int t = 0; t < 27; ++t) {
        const int mx = t / 9, my = (t / 3) % 3, mz = t % 3;
        const double dg = (2 - mx) * args.ix2 + (2 - my) * args.iy2 + (2 - mz) * args.iz2;
        // z = r / diag is formed in FP32; r.z uses the same rounded weights
        a.inv_diag_f[t] = dg > 0.0 ? float(1.0 / dg) : 0.f;
        a.inv_diag[t] = double(a.inv_diag_f[t]);
    }
    a.x = args.x;
    a.rhs = args.rhs;
    a.face0 = static_cast<float *>(args.r);
    a.face1 = static_cast<float *>(args.q);
    a.stop_rule = args.stop_rule;
    a.tol = args.tol; a.atol = args.atol; a.rtol = args.rtol;
    a.max_iters = args.max_iters;
    a.replace_every = args.replace_every > 0 ? args.replace_every : 50;
    if (cudaMalloc(&plan.partials, sizeof(double) * 2 * kResSlots * plan.grid) != cudaSuccess ||
        cudaMalloc(&plan.barrier, sizeof(GridBarrier)) != cudaSuccess) {
        pcg3d_res_destroy(plan);
        return false;
    }
    a.partials = plan.partials;
    a.bar = plan.barrier;
    plan.enabled = true;
    return true;
}

cudaError_t pcg3d_res_launch(const Pcg3dResPlan &plan, CgSeqState *state, cudaStream_t stream) {
    ResArgs a = plan.args;
    a.st = state;
    a.barrier_extra = take_injected_barrier_fault();
    a.spin_limit = a.barrier_extra ? kInjectedFaultSpinLimit : kBarrierSpinLimit;
    cudaError_t e = cudaMemsetAsync(plan.barrier, 0, sizeof(GridBarrier), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(state, 0, sizeof(CgSeqState), stream);
    void *params[] = {&a};
    if (e == cudaSuccess)
        e = cudaLaunchCooperativeKernel(plan.kernel, dim3(plan.grid), dim3(plan.block), params, plan.smem, stream);
    return e;
}

void pcg3d_res_destroy(Pcg3dResPlan &plan) {
    cudaFree(plan.partials);
    cudaFree(plan.barrier);
    plan = Pcg3dResPlan{};
}

}  // namespace flursys
