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
// the stencil pass: it forms d_new = z + beta d_old on the fly for its cells
// and their halo (bit-identical in every block) and writes d_new into the
// other half of a double buffer.
//
// One cooperative launch runs the whole solve. Two bounded grid barriers per
// iteration separate the reductions (d.q, then r.r / r.z / max|r|); every
// block reduces the per-block partials itself in a fixed order, so all blocks
// take bit-identical decisions and leave the loop together.
//
// Stencil passes walk tiles of 32 x 8 columns over a chunk of z planes
// ("2.5D" blocking): the current plane with its x/y halo sits in shared
// memory, the planes below and above in registers, so each vector element is
// read from memory about once per pass. Pointwise passes stream float4 /
// double2 vectors. 1/diag comes from a 27-entry table indexed by how many
// neighbours a cell misses in x, y and z (no divisions in the loop).
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

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "pcg3d.cuh"

namespace flursys {

namespace {

constexpr int TX = 32;
constexpr int TY = 8;
constexpr int kBlock = TX * TY;
constexpr int kNumPartials = 4;  // per block: [0] r.r  [1] r.z  [2] max|r|  [3] d.q / scratch

struct FastDiv;

struct Geo {
    int nx, ny, nz;
    int tiles_x, tiles_y, kc, chunks;  // tile decomposition of the stencil passes
    long long nxy, n;
    double ix2, iy2, iz2;
    unsigned long long div_row;  // FastDiv multiplier for nx / vector width
    unsigned long long div_nx;   // FastDiv multiplier for nx
    int vec;                     // nx is a multiple of the vector width
};

// Number of missing neighbours along one axis (0, 1 or 2).
__device__ __forceinline__ int miss(int i, int n) { return (i == 0) + (i == n - 1); }

template <typename V>
struct Vec4;
template <>
struct Vec4<float> {
    using T = float4;
};
template <>
struct Vec4<double> {
    using T = double2;
};

// Vectors written during this launch are read with plain (L1-cached) loads
// only after a grid barrier, whose acquire and fence make them visible.

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

struct SmemBase {
    double red[3 * (kBlock / 32)];  // up to two sums and a maximum per reduction
    double inv_diag[27];
    float inv_diag_f[27];
};

// Exact 32-bit division by a runtime constant (Lemire, Kaser and Kurz,
// "Faster remainder by direct computation", 2019): q = hi64(M * n) with
// M = floor((2^64 - 1) / d) + 1, valid for every 32-bit n and d.
struct FastDiv {
    unsigned long long m;
};
inline FastDiv make_fast_div(unsigned d) { return FastDiv{~0ull / d + 1ull}; }
__device__ __forceinline__ unsigned fast_div(const FastDiv &f, unsigned n) {
    return (unsigned)__umul64hi(f.m, (unsigned long long)n);
}

template <typename V, bool MIXED>
__global__ void __launch_bounds__(kBlock, 3) pcg3d_kernel(Pcg3dArgs a, Geo g) {
    __shared__ SmemBase sb;
    __shared__ double tile[(4 * TY + 2) * (TX + 2)];  // one plane with halo (FP64 or FP32 view)
    const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
    double *x = a.x;
    const double *__restrict__ rhs = a.rhs;
    V *r = static_cast<V *>(a.r);
    V *dbuf[2] = {static_cast<V *>(a.d0), static_cast<V *>(a.d1)};
    V *q = static_cast<V *>(a.q);
    float *dx = a.dx;  // MIXED only
    double *part = a.partials;
    GridBarrier *bar = a.barrier;
    // Grid barrier over the launch (plus a.barrier_extra arrivals that never
    // come when a test injects a barrier fault); a failure is recorded in the
    // result record before the block leaves.
    auto gsync = [&]() -> bool {
        return grid_sync_report(bar, gridDim.x + (unsigned)a.barrier_extra, &a.result->device_error, a.spin_limit);
    };
    const bool l2 = a.stop_rule == FLURSYS_STOP_REL_L2;
    const int nblk = gridDim.x;

    // 1/diag by missing-neighbour class 9*mx + 3*my + mz; a missing neighbour
    // count of 2 on one axis only occurs when that axis has one cell.
    if (threadIdx.x < 27) {
        const int mx = threadIdx.x / 9, my = (threadIdx.x / 3) % 3, mz = threadIdx.x % 3;
        const double dg = (2 - mx) * g.ix2 + (2 - my) * g.iy2 + (2 - mz) * g.iz2;
        sb.inv_diag[threadIdx.x] = dg > 0.0 ? 1.0 / dg : 0.0;
        sb.inv_diag_f[threadIdx.x] = float(sb.inv_diag[threadIdx.x]);
    }
    const unsigned char *row_class = a.row_class;  // 3*miss(j) + miss(k) per row (j, k)
    __syncthreads();
    const V *inv_diag_v = std::is_same<V, float>::value ? reinterpret_cast<const V *>(sb.inv_diag_f)
                                                       : reinterpret_cast<const V *>(sb.inv_diag);

    // ------------------------------------------------------------------
    // 2.5D stencil sweep over the block's tiles. A tile is TX columns by
    // TY*RY rows (each thread owns RY rows) by a chunk of planes. For a cell c:
    //   load(c)              issues the loads of the operand's raw inputs,
    //   make(raw, cls, pin)  forms the operand value (0 at the pinned cell),
    //   emit(c, cls, pin, v, Av) consumes (A v)_c (Av = v at the pinned cell).
    // cls indexes the 1/diag table. Raw inputs are prefetched two planes
    // ahead for the column and for the x/y halo, so the loads of a plane are
    // in flight while the two planes before it are computed.
    // ------------------------------------------------------------------
    auto stencil_pass = [&](auto ry_tag, auto load, auto make, auto emit) {
        constexpr int RY = decltype(ry_tag)::value;
        constexpr int TYR = TY * RY;
        constexpr int SW = TX + 2;
        using Raw = decltype(load(0));
        using T = decltype(make(load(0), 0, false));
        const T wx = T(g.ix2), wy = T(g.iy2), wz = T(g.iz2);
        const int nxy = g.nx * g.ny;
        const int tiles_y = (g.ny + TYR - 1) / TYR;
        const int ntiles = g.tiles_x * tiles_y * g.chunks;
        T *ts = reinterpret_cast<T *>(tile);
        const int h = threadIdx.x;
        const bool halo_thread = h < 2 * TX + 2 * TYR;
        for (int t = blockIdx.x; t < ntiles; t += nblk) {
            const int ch = t % g.chunks, col = t / g.chunks;
            const int i0 = (col % g.tiles_x) * TX, j0 = (col / g.tiles_x) * TYR;
            const int k0 = ch * g.kc, k1 = min(g.nz, k0 + g.kc);
            const int kmax = min(k1, g.nz - 1);  // last plane the columns read
            const int i = i0 + tx;
            const bool inx = i < g.nx;
            const T wxm = (inx && i > 0) ? wx : T(0), wxp = (inx && i + 1 < g.nx) ? wx : T(0);
            const int cx = 9 * miss(i, g.nx);
            int base[RY];
            bool in[RY];
#pragma unroll
            for (int m = 0; m < RY; ++m) {
                const int j = j0 + ty + m * TY;
                in[m] = inx && j < g.ny;
                base[m] = in[m] ? j * g.nx + i : 0;
            }
            int hi = 0, hj = 0;
            if (h < TX) { hi = i0 + h; hj = j0 - 1; }
            else if (h < 2 * TX) { hi = i0 + h - TX; hj = j0 + TYR; }
            else if (h < 2 * TX + TYR) { hi = i0 - 1; hj = j0 + h - 2 * TX; }
            else { hi = i0 + TX; hj = j0 + h - 2 * TX - TYR; }
            const bool hv = halo_thread && hi >= 0 && hi < g.nx && hj >= 0 && hj < g.ny;
            const int hbase = hv ? hj * g.nx + hi : 0;
            const int hcls = hv ? 9 * miss(hi, g.nx) + 3 * miss(hj, g.ny) : 0;
            const int hslot = halo_thread ? (hj - j0 + 1) * SW + (hi - i0 + 1) : 0;
            const bool hpcol = hv && hi == 0 && hj == 0;
            // prologue: below, cur, and two planes of lookahead
            T below[RY], cur[RY];
            Raw a1[RY], a2[RY], h1{}, h2{};
#pragma unroll
            for (int m = 0; m < RY; ++m) {
                below[m] = T(0);
                cur[m] = T(0);
                a1[m] = Raw{};
                a2[m] = Raw{};
                if (in[m]) {
                    const int cxy = cx + 3 * miss(j0 + ty + m * TY, g.ny);
                    const bool pc = base[m] == 0;
                    if (k0 > 0) below[m] = make(load(base[m] + (k0 - 1) * nxy), cxy + miss(k0 - 1, g.nz), false);
                    cur[m] = make(load(base[m] + k0 * nxy), cxy + miss(k0, g.nz), pc && k0 == 0);
                    if (k0 + 1 <= kmax) a1[m] = load(base[m] + (k0 + 1) * nxy);
                    if (k0 + 2 <= kmax) a2[m] = load(base[m] + (k0 + 2) * nxy);
                }
            }
            if (hv) {
                h1 = load(hbase + k0 * nxy);
                if (k0 + 1 < k1) h2 = load(hbase + (k0 + 1) * nxy);
            }
            for (int k = k0; k < k1; ++k) {
                const int mk = miss(k, g.nz);
                T above[RY];
#pragma unroll
                for (int m = 0; m < RY; ++m) {
                    above[m] = T(0);
                    if (in[m]) {
                        if (k + 1 < g.nz)
                            above[m] = make(a1[m], cx + 3 * miss(j0 + ty + m * TY, g.ny) + miss(k + 1, g.nz), false);
                        a1[m] = a2[m];
                        if (k + 3 <= kmax) a2[m] = load(base[m] + (k + 3) * nxy);
                    }
                }
                T hval = T(0);
                if (hv) {
                    hval = make(h1, hcls + mk, hpcol && k == 0);
                    h1 = h2;
                    if (k + 2 < k1) h2 = load(hbase + (k + 2) * nxy);
                }
#pragma unroll
                for (int m = 0; m < RY; ++m) ts[(ty + m * TY + 1) * SW + tx + 1] = cur[m];
                if (halo_thread) ts[hslot] = hval;
                __syncthreads();
                const T wzm = k > 0 ? wz : T(0), wzp = k + 1 < g.nz ? wz : T(0);
#pragma unroll
                for (int m = 0; m < RY; ++m) {
                    if (in[m]) {
                        const int j = j0 + ty + m * TY;
                        const T wym = j > 0 ? wy : T(0), wyp = j + 1 < g.ny ? wy : T(0);
                        const int sp = (ty + m * TY + 1) * SW + tx + 1;
                        const T ax = (wxm + wxp + wym + wyp + wzm + wzp) * cur[m] -
                                     (wxm * ts[sp - 1] + wxp * ts[sp + 1] + wym * ts[sp - SW] + wyp * ts[sp + SW] +
                                      wzm * below[m] + wzp * above[m]);
                        const bool pin = base[m] == 0 && k == 0;
                        emit(base[m] + k * nxy, cx + 3 * miss(j, g.ny) + mk, pin, cur[m], pin ? cur[m] : ax);
                    }
                }
                __syncthreads();
#pragma unroll
                for (int m = 0; m < RY; ++m) {
                    below[m] = cur[m];
                    cur[m] = above[m];
                }
            }
        }
    };
    constexpr int kRyA = 1;  // rows per thread, operand passes
    using RyA = std::integral_constant<int, kRyA>;
    using RyX = std::integral_constant<int, 1>;  // FP64 residual passes

    const long long tid0 = (long long)blockIdx.x * kBlock + threadIdx.x;
    const long long stride = (long long)nblk * kBlock;

    // r.r, r.z and max|r| through one set of block barriers (the same
    // shuffle tree per value as separate reductions)
    auto write_partials3 = [&](double srr, double srz, double smax) {
        double t[2] = {srr, srz};
        block_reduce_n<kBlock, 2, true>(t, smax, sb.red);
        if (threadIdx.x == 0) {
            part[blockIdx.x * kNumPartials + 0] = t[0];
            part[blockIdx.x * kNumPartials + 1] = t[1];
            part[blockIdx.x * kNumPartials + 2] = smax;
        }
    };
    auto reduce3 = [&](double &rr, double &rz, double &rmax) {
        double t[2] = {0.0, 0.0};
        double s2 = 0.0;
        for (int b = threadIdx.x; b < nblk; b += kBlock) {
            t[0] += part[b * kNumPartials + 0];
            t[1] += part[b * kNumPartials + 1];
            s2 = fmax(s2, part[b * kNumPartials + 2]);
        }
        block_reduce_n<kBlock, 2, true>(t, s2, sb.red);
        rr = t[0];
        rz = t[1];
        rmax = s2;
    };
    auto reduce_slot3 = [&]() -> double {
        double s = 0.0;
        for (int b = threadIdx.x; b < nblk; b += kBlock) s += part[b * kNumPartials + 3];
        return block_sum<kBlock>(s, sb.red);
    };

    // r = b - A x in FP64 (b = -rhs), stored in V; optional zeroing of dx.
    auto load_x = [&](int c) -> double { return x[c]; };
    auto make_x = [&](double v, int, bool pin) -> double { return pin ? 0.0 : v; };
    auto residual_pass = [&](bool zero_dx) {
        double srr = 0.0, srz = 0.0, smax = 0.0;
        stencil_pass(RyX{}, load_x, make_x, [&](int c, int cls, bool pin, double, double ax) {
            const double rr = pin ? 0.0 : -__ldg(rhs + c) - ax;
            const V rv = V(rr);
            r[c] = rv;
            if (MIXED && zero_dx) dx[c] = 0.f;
            const double rd = double(rv);
            srr += rd * rd;
            srz += rd * rd * (pin ? 1.0 : sb.inv_diag[cls]);
            smax = fmax(smax, fabs(rd));
        });
        write_partials3(srr, srz, smax);
    };
    auto fold = [&]() {  // x += dx (MIXED)
        for (int c = (int)tid0; c < (int)g.n; c += (int)stride) {
            if (c == 0) { x[0] = 0.0; continue; }
            x[c] += double(dx[c]);
        }
    };

    int status = FLURSYS_LINEAR_MAX_ITERATIONS;
    int error = 0;
    long long iterations = 0;
    double residual = 0.0, initial = 0.0, threshold = 0.0;

    if (blockIdx.x == 0 && threadIdx.x == 0) x[0] = 0.0;
    residual_pass(true);
    if (!gsync()) return;
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

    unsigned long long tph[4] = {0, 0, 0, 0};
    unsigned long long tmark = gtimer();
    auto lap = [&](int slot) {
        const unsigned long long now = gtimer();
        tph[slot] += now - tmark;
        tmark = now;
    };
    for (long long it = 0; !done && it < a.max_iters; ++it) {
        iterations = it + 1;
        V *dcur = dbuf[it & 1];
        const V *dold = dbuf[(it + 1) & 1];
        // ---- phase A: d = z + beta d_old (cells + halo), q = A d, partial d.q ----
        double sdq = 0.0;
        const V vbeta = V(beta);
        struct RawA {
            V r, d;
        };
        auto load_a = [&](int c) -> RawA { return RawA{r[c], first ? V(0) : dold[c]}; };
        auto make_a = [&](RawA v, int cls, bool pin) -> V {
            if (pin) return V(0);
            const V z = v.r * inv_diag_v[cls];
            return first ? z : V(z + vbeta * v.d);
        };
        stencil_pass(RyA{}, load_a, make_a, [&](int c, int, bool, V dc, V qc) {
            dcur[c] = dc;
            q[c] = qc;
            sdq += double(dc) * double(qc);
        });
        lap(0);
        {
            const double t = block_sum<kBlock>(sdq, sb.red);
            if (threadIdx.x == 0) part[blockIdx.x * kNumPartials + 3] = t;
        }
        if (!gsync()) return;
        const double dq = reduce_slot3();
        lap(2);
        if (fabs(dq) < 1.0e-30 || !isfinite(dq)) { error = FLURSYS_ERR_BREAKDOWN; break; }
        const double alpha = rz_old / dq;
        if (!isfinite(alpha)) { error = FLURSYS_ERR_BREAKDOWN; break; }
        // ---- phase B: x += alpha d, r -= alpha q, partial r.r, r.z, max|r| ----
        double srr = 0.0, srz = 0.0, smax = 0.0;
        {
            using V4 = typename Vec4<V>::T;
            constexpr int W = sizeof(V4) / sizeof(V);
            const int nrow = g.nx / W;  // vectors per row when g.vec
            const int nv = g.vec ? g.ny * g.nz * nrow : 0;
            for (int cv = (int)tid0; cv < nv; cv += (int)stride) {
                const int row = (int)fast_div(FastDiv{g.div_row}, (unsigned)cv);
                const int i0 = (cv - row * nrow) * W;
                const int c0 = cv * W;
                const int rcls = row_class[row];
                const V4 d4 = reinterpret_cast<const V4 *>(dcur)[cv];
                const V4 q4 = reinterpret_cast<const V4 *>(q)[cv];
                V4 r4 = reinterpret_cast<const V4 *>(r)[cv];
                const V *dv = reinterpret_cast<const V *>(&d4);
                const V *qv = reinterpret_cast<const V *>(&q4);
                V *rv = reinterpret_cast<V *>(&r4);
                if (MIXED) {
                    float4 x4 = reinterpret_cast<const float4 *>(dx)[cv];
                    float *xv = reinterpret_cast<float *>(&x4);
#pragma unroll
                    for (int e = 0; e < W; ++e) xv[e] = float(double(xv[e]) + alpha * double(dv[e]));
                    reinterpret_cast<float4 *>(dx)[cv] = x4;
                } else {
                    double2 *xp = reinterpret_cast<double2 *>(x + c0);
                    double2 x2 = *xp;
                    x2.x += (c0 == 0) ? 0.0 : alpha * double(dv[0]);
                    x2.y += alpha * double(dv[1]);
                    *xp = x2;
                }
                // interior cells share one 1/diag; the end cells of a row may differ
                const double idg_mid = sb.inv_diag[rcls];
#pragma unroll
                for (int e = 0; e < W; ++e) {
                    rv[e] = V(double(rv[e]) - alpha * double(qv[e]));
                    const double rd = double(rv[e]);
                    const int ie = i0 + e;
                    const double idg = (ie == 0 || ie == g.nx - 1) ? sb.inv_diag[9 * miss(ie, g.nx) + rcls] : idg_mid;
                    srr += rd * rd;
                    srz += rd * rd * ((c0 + e == 0) ? 1.0 : idg);
                    smax = fmax(smax, fabs(rd));
                }
                reinterpret_cast<V4 *>(r)[cv] = r4;
            }
            const int ns = g.vec ? 0 : (int)g.n;  // scalar path when nx is not a multiple of W
            for (int c = (int)tid0; c < ns; c += (int)stride) {
                const int row = (int)fast_div(FastDiv{g.div_nx}, (unsigned)c);
                const int i = c - row * g.nx;
                const double dcv = double(dcur[c]);
                if (MIXED) dx[c] = float(double(dx[c]) + alpha * dcv);
                else if (c != 0) x[c] += alpha * dcv;
                const V rv = V(double(r[c]) - alpha * double(q[c]));
                r[c] = rv;
                const double rd = double(rv);
                srr += rd * rd;
                srz += rd * rd * (c == 0 ? 1.0 : sb.inv_diag[9 * miss(i, g.nx) + row_class[row]]);
                smax = fmax(smax, fabs(rd));
            }
        }
        lap(1);
        write_partials3(srr, srz, smax);
        if (!gsync()) return;
        double rz_new;
        reduce3(rr, rz_new, rmax);
        lap(2);
        residual = l2 ? sqrt(rr) : rmax;
        if (!isfinite(residual)) { error = FLURSYS_ERR_NON_FINITE; break; }
        bool conv = l2 ? (residual <= threshold) : (residual < threshold);
        if (MIXED && (conv || ((it + 1) % a.replace_every) == 0)) {
            fold();
            if (!gsync()) return;
            residual_pass(true);
            if (!gsync()) return;
            reduce3(rr, rz_new, rmax);
            residual = l2 ? sqrt(rr) : rmax;
            if (!isfinite(residual)) { error = FLURSYS_ERR_NON_FINITE; break; }
            conv = l2 ? (residual <= threshold) : (residual < threshold);
            lap(3);
        }
        if (conv) { status = FLURSYS_LINEAR_CONVERGED; break; }
        if (fabs(rz_old) < 1.0e-30) break;
        beta = rz_new / rz_old;
        rz_old = rz_new;
        first = false;
    }

    if (MIXED && error == 0 && status != FLURSYS_LINEAR_CONVERGED) fold();
    if (!gsync()) return;
    // ---- final FP64 check: ||b - A x||_2 of the solution in HBM ----
    double s_true = 0.0;
    stencil_pass(RyX{}, load_x, make_x, [&](int c, int, bool pin, double, double ax) {
        const double t = pin ? 0.0 : -__ldg(rhs + c) - ax;
        s_true += t * t;
    });
    {
        const double t = block_sum<kBlock>(s_true, sb.red);
        if (threadIdx.x == 0) part[blockIdx.x * kNumPartials + 3] = t;
    }
    if (!gsync()) return;
    const double true_rr = reduce_slot3();
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
        for (int p = 0; p < 4; ++p) res->phase_ns[p] = tph[p];
        res->phase_ns[4] = res->phase_ns[5] = 0;
    }
}

Geo make_geo(const Pcg3dArgs &a, int grid) {
    Geo g{};
    g.nx = a.nx; g.ny = a.ny; g.nz = a.nz;
    g.nxy = (long long)a.nx * a.ny;
    g.n = g.nxy * a.nz;
    g.ix2 = a.ix2; g.iy2 = a.iy2; g.iz2 = a.iz2;
    const int ry = 1;  // rows per thread of the operand pass
    g.tiles_x = (a.nx + TX - 1) / TX;
    g.tiles_y = (a.ny + TY * ry - 1) / (TY * ry);
    const long long cols = (long long)g.tiles_x * g.tiles_y;
    // About eight tiles per block, at least four planes per tile.
    long long want = std::max(1LL, (long long)grid * 8 / std::max(1LL, cols));
    int kc = (int)std::max(4LL, (a.nz + want - 1) / want);
    kc = std::min(kc, a.nz);
    g.kc = kc;
    g.chunks = (a.nz + kc - 1) / kc;
    const int w = a.precision_vec_width > 0 ? a.precision_vec_width : 1;
    g.vec = (a.nx % w) == 0;
    g.div_row = make_fast_div((unsigned)std::max(1, a.nx / w)).m;
    g.div_nx = make_fast_div((unsigned)a.nx).m;
    return g;
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

cudaError_t pcg3d_make_row_class(int ny, int nz, unsigned char **out, cudaStream_t stream) {
    std::vector<unsigned char> h((size_t)ny * nz);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j) h[(size_t)k * ny + j] = (unsigned char)(3 * ((j == 0) + (j == ny - 1)) + ((k == 0) + (k == nz - 1)));
    cudaError_t e = cudaMalloc(out, h.size());
    if (e == cudaSuccess) e = cudaMemcpyAsync(*out, h.data(), h.size(), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    return e;
}

int pcg3d_block_size() { return kBlock; }
int pcg3d_num_partials() { return kNumPartials; }

cudaError_t pcg3d_launch(const Pcg3dArgs &args, int grid, int precision, cudaStream_t stream) {
    Pcg3dArgs a = args;
    a.barrier_extra = take_injected_barrier_fault();
    a.spin_limit = a.barrier_extra ? kInjectedFaultSpinLimit : kBarrierSpinLimit;
    Geo g = make_geo(args, grid);
    void *params[] = {&a, &g};
    if (precision == FLURSYS_PRECISION_MIXED)
        return cudaLaunchCooperativeKernel((const void *)pcg3d_kernel<float, true>, dim3(grid), dim3(kBlock),
                                           params, 0, stream);
    return cudaLaunchCooperativeKernel((const void *)pcg3d_kernel<double, false>, dim3(grid), dim3(kBlock),
                                       params, 0, stream);
}

}  // namespace flursys
