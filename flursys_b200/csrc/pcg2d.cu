// pcg2d.cu — persistent pressure solvers of the 2D structured solver
// (src/solver/incompressible.rs), batched over independent instances.
//
// PCG follows solve_pressure_pcg (:1048-1214) with the operator of
// apply_pressure_operator (:1216-1255): fluid rows sum over in-range,
// non-solid neighbours; solid and pressure-outlet cells are identity rows
// holding 0 or the outlet pressure. Without a pressure outlet the system is
// pure Neumann and x, b, r, z and d are projected to zero mean over the fluid
// cells as in project_zero_mean (:2338-2377). The projections are folded into
// the passes that produce each vector:
//   pass 1  d = (z - mean z) + beta (d_old - mean d_old) on the fly, q = A d,
//           sums d.q, sum q, sum d      -> barrier -> mean d, d.q, alpha
//   pass 2  x += alpha d, r -= alpha q, sums x, r       -> barrier -> means
//   pass 3  x, r projected and stored, stop residual, z = r/diag stored,
//           sums z, r.z, r              -> barrier -> residual, mean z, rz
// Since A annihilates the fluid indicator, A(d - m) = A d and
// d'.q = d.q - m sum q, so each projected quantity equals the reference's up
// to rounding. With an outlet, passes 2 and 3 merge (two barriers).
//
// SOR follows solve_pressure_sor (:979-1046) with red-black ordering (not
// iterate-identical to the reference's lexicographic sweep), the reference
// cell shift of :1024-1035 and the stop test of pressure_residual
// (:1532-1567).
//
// Every barrier wait is bounded (common.cuh); all blocks of an instance
// reduce the same partials in the same order and leave their loops together.
#include <cuda_runtime.h>

#include <cmath>

#include "common.cuh"
#include "pcg2d.cuh"

namespace flursys {

namespace {

constexpr int kBlock = 256;
// Partial-sum columns per block: two sets of kRoundCols that alternate by
// reduction round, so that a block never overwrites a set that a slower
// block may still be reading (the next write to the same set is one
// barrier further on).
constexpr int kRoundCols = 8;
constexpr int kParts = 2 * kRoundCols;
constexpr int kU = 4;  // cells per thread per step of the plain-operator passes

// Barriers between the passes of one instance. GridSync: the bounded
// software grid barrier over the instance's blocks. ClusterSync: the
// instance runs as one thread-block cluster and the passes are separated by
// the hardware cluster barrier (release / acquire at cluster scope, so
// everything written before it is visible after it in every block of the
// cluster). Either way the blocks' partial sums meet in global memory, read
// through L2. (Partials in distributed shared memory measured no faster on
// the 128^2 cavity and need a closing barrier to keep every block's shared
// memory alive until the last read.)
struct GridSync {
    GridBarrier *bar;
    unsigned nb;
    double *partials;
    unsigned *report;  // the instance's PcgResultDev::device_error
    __device__ __forceinline__ bool operator()() const { return grid_sync_report(bar, nb, report); }
    __device__ __forceinline__ void put(int lb, int col, double v) const { partials[lb * kParts + col] = v; }
    __device__ __forceinline__ double get(int b, int col) const { return __ldcg(partials + b * kParts + col); }
};
struct ClusterSync {
    double *partials;
    __device__ __forceinline__ bool operator()() const {
        asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
        return true;
    }
    __device__ __forceinline__ void put(int lb, int col, double v) const { partials[lb * kParts + col] = v; }
    __device__ __forceinline__ double get(int b, int col) const { return __ldcg(partials + b * kParts + col); }
};

__device__ __forceinline__ bool solid(const uint8_t *f, int c) { return (f[c] & kCellSolid) != 0; }
__device__ __forceinline__ bool ident(const uint8_t *f, int c) { return (f[c] & 3) != 0; }

struct Ctx {
    Pcg2dInstance in;
    int lb;  // block index within the instance
    int n, c_begin, c_end;
    int step_i, step_j;  // kBlock cells = step_j rows + step_i columns
    int round;           // reduction rounds completed (selects the column set)
};

// A thread's walk over the cells of its block: c advances by kBlock and
// (i, j) follow without a division per cell.
struct CellIter {
    int c, i, j;
};
__device__ __forceinline__ CellIter first_cell(const Ctx &k) {
    const int c = k.c_begin + (int)threadIdx.x;
    return CellIter{c, c % k.in.nx, c / k.in.nx};
}
__device__ __forceinline__ void next_cell(const Ctx &k, CellIter &it) {
    it.c += kBlock;
    it.i += k.step_i;
    it.j += k.step_j;
    if (it.i >= k.in.nx) {
        it.i -= k.in.nx;
        ++it.j;
    }
}

// Diagonal of a fluid row.
__device__ __forceinline__ double diag2(const Ctx &k, int c, int i, int j) {
    const uint8_t *f = k.in.flags;
    double d = 0.0;
    if (i + 1 < k.in.nx && !solid(f, c + 1)) d += k.in.idx2;
    if (i > 0 && !solid(f, c - 1)) d += k.in.idx2;
    if (j + 1 < k.in.ny && !solid(f, c + k.in.nx)) d += k.in.idy2;
    if (j > 0 && !solid(f, c - k.in.nx)) d += k.in.idy2;
    return d;
}

// (A v)_c for a fluid row with `val(nb)` giving the operand.
template <typename T, typename F>
__device__ __forceinline__ T apply_row(const Ctx &k, int c, int i, int j, T vc, F val) {
    const uint8_t *f = k.in.flags;
    const T wx = T(k.in.idx2), wy = T(k.in.idy2);
    T dg = T(0), s = T(0);
    if (i + 1 < k.in.nx && !solid(f, c + 1)) { dg += wx; s += wx * val(c + 1); }
    if (i > 0 && !solid(f, c - 1)) { dg += wx; s += wx * val(c - 1); }
    if (j + 1 < k.in.ny && !solid(f, c + k.in.nx)) { dg += wy; s += wy * val(c + k.in.nx); }
    if (j > 0 && !solid(f, c - k.in.nx)) { dg += wy; s += wy * val(c - k.in.nx); }
    return dg * vc - s;
}

// Block partial sums of NV values into columns 0..NV-1 of this round's set.
template <int NV, typename Sync>
__device__ __forceinline__ void write_parts(const Ctx &k, const Sync &sync, double (&v)[NV], double *red) {
    block_sum_n<kBlock, NV>(v, red);
    const int base = (k.round & 1) * kRoundCols;
    if (threadIdx.x == 0)
#pragma unroll
        for (int p = 0; p < NV; ++p) sync.put(k.lb, base + p, v[p]);
}
// Sums over the instance's blocks of columns 0..NV-1, in block order.
template <int NV, typename Sync>
__device__ __forceinline__ void read_sums(Ctx &k, const Sync &sync, double (&out)[NV], double *red) {
    const int base = (k.round & 1) * kRoundCols;
#pragma unroll
    for (int p = 0; p < NV; ++p) out[p] = 0.0;
    for (int b = threadIdx.x; b < k.in.nblocks; b += kBlock)
#pragma unroll
        for (int p = 0; p < NV; ++p) out[p] += sync.get(b, base + p);
    block_sum_n<kBlock, NV>(out, red);
    ++k.round;
}
// write_parts plus the block maximum of mx into column NV.
template <int NV, typename Sync>
__device__ __forceinline__ void write_parts_max(const Ctx &k, const Sync &sync, double (&v)[NV], double mx,
                                                double *red) {
    block_reduce_n<kBlock, NV, true>(v, mx, red);
    const int base = (k.round & 1) * kRoundCols;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int p = 0; p < NV; ++p) sync.put(k.lb, base + p, v[p]);
        sync.put(k.lb, base + NV, mx);
    }
}
// read_sums plus the maximum over blocks of column NV.
template <int NV, typename Sync>
__device__ __forceinline__ void read_sums_max(Ctx &k, const Sync &sync, double (&out)[NV], double &mx, double *red) {
    const int base = (k.round & 1) * kRoundCols;
#pragma unroll
    for (int p = 0; p < NV; ++p) out[p] = 0.0;
    mx = 0.0;
    for (int b = threadIdx.x; b < k.in.nblocks; b += kBlock) {
#pragma unroll
        for (int p = 0; p < NV; ++p) out[p] += sync.get(b, base + p);
        mx = fmax(mx, sync.get(b, base + NV));
    }
    block_reduce_n<kBlock, NV, true>(out, mx, red);
    ++k.round;
}
template <typename Sync>
__device__ __forceinline__ void write_max(const Ctx &k, const Sync &sync, double v, double *red) {
    const double t = block_max<kBlock>(v, red);
    if (threadIdx.x == 0) sync.put(k.lb, (k.round & 1) * kRoundCols, t);
}
template <typename Sync>
__device__ __forceinline__ double read_max(Ctx &k, const Sync &sync, double *red) {
    const int col = (k.round & 1) * kRoundCols;
    double s = 0.0;
    for (int b = threadIdx.x; b < k.in.nblocks; b += kBlock) s = fmax(s, sync.get(b, col));
    ++k.round;
    return block_max<kBlock>(s, red);
}

template <typename V, bool MIXED, typename Sync>
__device__ void pcg_instance(Ctx &k, double *red, const Sync &sync) {
    const Pcg2dInstance &in = k.in;
    const uint8_t *f = in.flags;
    double *x = in.x;
    V *r = static_cast<V *>(in.r);
    V *z = static_cast<V *>(in.z);
    V *dbuf[2] = {static_cast<V *>(in.d0), static_cast<V *>(in.d1)};
    V *q = static_cast<V *>(in.q);
    const bool proj = in.project != 0;
    const bool l2 = in.stop_rule == FLURSYS_STOP_REL_L2;
    const double cnt = in.count_fluid > 0 ? double(in.count_fluid) : 1.0;
    const int nx = in.nx;
    // no solid or outlet cell: every row is a fluid row of the plain
    // 5-point operator, so the passes skip the flag bytes
    const bool plain = in.count_fluid == (long long)in.nx * in.ny;
    const int lane = threadIdx.x & 31;
    auto bval = [&](int c) -> double {  // b of the system (before projection)
        const uint8_t fc = f[c];
        if (fc & kCellOutlet) return in.outlet_pressure;
        if (fc & kCellSolid) return 0.0;
        return -__ldg(in.rhs + c);
    };

    int status = FLURSYS_LINEAR_MAX_ITERATIONS, error = 0;
    long long iterations = 0;
    double residual = 0.0, initial = 0.0, initial_l2 = 0.0, threshold = 0.0;
    double mb = 0.0;  // mean of b over fluid cells (pure Neumann)
    double rz_old = 0.0, mz = 0.0;

    // ---- I1: identity rows take their fixed values; sums of x and b ----
    {
        double sx = 0.0, sb = 0.0;
        for (int c = k.c_begin + threadIdx.x; c < k.c_end; c += kBlock) {
            const uint8_t fc = f[c];
            if (fc & 3) {
                x[c] = (fc & kCellOutlet) ? in.outlet_pressure : 0.0;
            } else {
                sx += x[c];
                sb += bval(c);
            }
        }
        double v[2] = {sx, sb};
        write_parts<2>(k, sync, v, red);
    }
    if (!sync()) return;
    double m0[2];
    read_sums<2>(k, sync, m0, red);
    double mx = proj ? m0[0] / cnt : 0.0;
    mb = proj ? m0[1] / cnt : 0.0;
    if (proj) {
        for (int c = k.c_begin + threadIdx.x; c < k.c_end; c += kBlock)
            if (!ident(f, c)) x[c] -= mx;
        if (!sync()) return;
    }

    // ---- r = b' - A x (FP64), projected; residual; z; r.z ----
    auto residual_pass = [&]() -> bool {
        double sr = 0.0;
        for (CellIter it = first_cell(k); it.c < k.c_end; next_cell(k, it)) {
            const int c = it.c, i = it.i, j = it.j;
            double rv = 0.0;
            if (!ident(f, c)) {
                rv = bval(c) - mb - apply_row<double>(k, c, i, j, x[c], [&](int m) { return x[m]; });
                sr += rv;
            }
            r[c] = V(rv);
        }
        double v[1] = {sr};
        write_parts<1>(k, sync, v, red);
        if (!sync()) return false;
        double m1[1];
        read_sums<1>(k, sync, m1, red);
        const double mr = proj ? m1[0] / cnt : 0.0;
        double s_rr = 0.0, s_max = 0.0, s_z = 0.0, s_rz = 0.0, s_r = 0.0;
        for (CellIter it = first_cell(k); it.c < k.c_end; next_cell(k, it)) {
            const int c = it.c, i = it.i, j = it.j;
            double rv = double(r[c]);
            double zv = rv;
            if (!ident(f, c)) {
                if (proj) {
                    rv = double(V(rv - mr));
                    r[c] = V(rv);
                }
                const double dg = diag2(k, c, i, j);
                zv = dg > 0.0 ? rv / dg : rv;
                s_z += zv;
                s_r += rv;
            }
            z[c] = V(zv);
            s_rr += rv * rv;
            s_max = fmax(s_max, fabs(rv));
            s_rz += rv * double(V(zv));
        }
        double v2[4] = {s_rr, s_z, s_rz, s_r};
        write_parts_max<4>(k, sync, v2, s_max, red);
        return sync();
    };
    // Sums of the projected residual and solution over fluid cells, carried
    // from one iteration to the next: the means that the projection of the
    // updated x and r removes follow from them without another reduction,
    //   sum(x + a (d - md)) = sum x,   sum(r - a q) = sum r - a sum q.
    double s_r_prev = 0.0, s_x_prev = 0.0;
    auto read_residual_sums = [&](double &rr, double &rmax, double &rz) {
        double s4[4];
        read_sums_max<4>(k, sync, s4, rmax, red);
        rr = s4[0];
        const double sz = s4[1], srz = s4[2], sr = s4[3];
        mz = proj ? sz / cnt : 0.0;
        rz = srz - mz * sr;  // r'.(z - mean z)
        s_r_prev = sr;
    };
    s_x_prev = m0[0] - cnt * mx;  // sum of x after the initial projection
    if (!residual_pass()) return;
    double rr, rmax;
    read_residual_sums(rr, rmax, rz_old);
    initial_l2 = sqrt(rr);
    initial = l2 ? initial_l2 : rmax;
    threshold = l2 ? in.atol + in.rtol * initial : in.tol;
    residual = initial;
    bool done = l2 ? (residual <= threshold) : (residual < threshold);
    if (done) status = FLURSYS_LINEAR_CONVERGED;
    double beta = 0.0, md_old = 0.0;
    bool first = true;

    for (long long it = 0; !done && it < in.max_iters; ++it) {
        iterations = it + 1;
        V *dcur = dbuf[it & 1];
        const V *dold = dbuf[(it + 1) & 1];
        // ---- pass 1: direction + stencil ----
        auto dn = [&](int m) -> V {
            if (ident(f, m)) return V(0);
            const double zm = double(z[m]) - mz;
            return first ? V(zm) : V(zm + beta * (double(dold[m]) - md_old));
        };
        double s_dq = 0.0, s_q = 0.0, s_d = 0.0;
        if (plain) {
            // U cells per thread per step, every load issued before use; x
            // neighbours by shuffle (lanes hold consecutive cells), lane 0 /
            // lane 31 and the range tail load theirs
            const V wxv = V(in.idx2), wyv = V(in.idy2);
            auto dpl = [&](int m) -> V {
                const double zm = double(z[m]) - mz;
                return first ? V(zm) : V(zm + beta * (double(dold[m]) - md_old));
            };
            CellIter it = first_cell(k);
            while (__any_sync(0xffffffffu, it.c < k.c_end)) {
                CellIter cs[kU];
                V dc[kU], dN[kU], dS[kU], dE[kU], dW[kU];
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    cs[u] = it;
                    const bool ok = it.c < k.c_end;
                    const int c = ok ? it.c : k.c_end - 1;
                    const int i = ok ? it.i : 0, j = ok ? it.j : 0;
                    dc[u] = dpl(c);
                    dN[u] = ok && j + 1 < in.ny ? dpl(c + nx) : V(0);
                    dS[u] = ok && j > 0 ? dpl(c - nx) : V(0);
                    const bool own_e = lane < 31 && it.c + 1 < k.c_end;
                    dE[u] = ok && !own_e && i + 1 < nx ? dpl(c + 1) : V(0);
                    dW[u] = ok && lane == 0 && i > 0 ? dpl(c - 1) : V(0);
                    next_cell(k, it);
                }
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const V e_sh = __shfl_down_sync(0xffffffffu, dc[u], 1);
                    const V w_sh = __shfl_up_sync(0xffffffffu, dc[u], 1);
                    const int c = cs[u].c, i = cs[u].i, j = cs[u].j;
                    if (c >= k.c_end) continue;
                    const V east = (lane < 31 && c + 1 < k.c_end) ? e_sh : dE[u];
                    const V west = lane > 0 ? w_sh : dW[u];
                    V dg = V(0), sn = V(0);
                    if (i + 1 < nx) { dg += wxv; sn += wxv * east; }
                    if (i > 0) { dg += wxv; sn += wxv * west; }
                    if (j + 1 < in.ny) { dg += wyv; sn += wyv * dN[u]; }
                    if (j > 0) { dg += wyv; sn += wyv * dS[u]; }
                    const V qc = dg * dc[u] - sn;
                    dcur[c] = dc[u];
                    q[c] = qc;
                    s_q += double(qc);
                    s_d += double(dc[u]);
                    s_dq += double(dc[u]) * double(qc);
                }
            }
        } else {
            for (CellIter it = first_cell(k); it.c < k.c_end; next_cell(k, it)) {
                const int c = it.c, i = it.i, j = it.j;
                const V dc = dn(c);
                V qc = dc;
                if (!ident(f, c)) {
                    qc = apply_row<V>(k, c, i, j, dc, dn);
                    s_q += double(qc);
                    s_d += double(dc);
                }
                dcur[c] = dc;
                q[c] = qc;
                s_dq += double(dc) * double(qc);
            }
        }
        {
            double v[3] = {s_dq, s_q, s_d};
            write_parts<3>(k, sync, v, red);
        }
        if (!sync()) return;
        double s3[3];
        read_sums<3>(k, sync, s3, red);
        const double sdq = s3[0];
        const double md = proj ? s3[2] / cnt : 0.0;
        const double dq = proj ? sdq - md * s3[1] : sdq;
        if (fabs(dq) < 1.0e-30 || !isfinite(dq)) { error = FLURSYS_ERR_BREAKDOWN; break; }
        const double alpha = rz_old / dq;
        if (!isfinite(alpha)) { error = FLURSYS_ERR_BREAKDOWN; break; }
        // ---- the means removed by the projection of the updated x and r ----
        double mr = 0.0;
        if (proj) {
            mx = s_x_prev / cnt;
            mr = (s_r_prev - alpha * s3[1]) / cnt;
        }
        // ---- pass 2: update, projection, residual, z, r.z ----
        // x += a (d - md) and r -= a q (FP32 r rounded as stored), then the
        // means are removed: the arithmetic of an update pass followed by a
        // projection pass, in one sweep.
        double s_rr = 0.0, s_max = 0.0, s_z = 0.0, s_rz = 0.0, s_r = 0.0, s_x = 0.0;
        if (plain) {
            for (CellIter it = first_cell(k); it.c < k.c_end;) {
                CellIter cs[kU];
                double xv[kU], pv[kU];
                V rv0[kU], qv[kU];
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    cs[u] = it;
                    const bool ok = it.c < k.c_end;
                    const int c = ok ? it.c : k.c_begin;
                    xv[u] = x[c];
                    rv0[u] = r[c];
                    pv[u] = double(dcur[c]);
                    qv[u] = q[c];
                    next_cell(k, it);
                }
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const int c = cs[u].c, i = cs[u].i, j = cs[u].j;
                    if (c >= k.c_end) continue;
                    double rv;
                    if (proj) {
                        const double xn = (xv[u] + alpha * (pv[u] - md)) - mx;
                        x[c] = xn;
                        s_x += xn;
                        rv = double(V(double(V(double(rv0[u]) - alpha * double(qv[u]))) - mr));
                    } else {
                        x[c] = xv[u] + alpha * pv[u];
                        rv = double(V(double(rv0[u]) - alpha * double(qv[u])));
                    }
                    r[c] = V(rv);
                    double dg = 0.0;
                    if (i + 1 < nx) dg += in.idx2;
                    if (i > 0) dg += in.idx2;
                    if (j + 1 < in.ny) dg += in.idy2;
                    if (j > 0) dg += in.idy2;
                    const double zv = dg > 0.0 ? rv / dg : rv;
                    s_z += zv;
                    s_r += rv;
                    z[c] = V(zv);
                    s_rr += rv * rv;
                    s_max = fmax(s_max, fabs(rv));
                    s_rz += rv * double(V(zv));
                }
            }
        } else
        for (CellIter it = first_cell(k); it.c < k.c_end; next_cell(k, it)) {
            const int c = it.c, i = it.i, j = it.j;
            double rv;
            double zv;
            if (ident(f, c)) {
                rv = double(r[c]);
                zv = rv;
            } else {
                if (proj) {
                    const double xn = (x[c] + alpha * (double(dcur[c]) - md)) - mx;
                    x[c] = xn;
                    s_x += xn;
                    rv = double(V(double(V(double(r[c]) - alpha * double(q[c]))) - mr));
                } else {
                    x[c] += alpha * double(dcur[c]);
                    rv = double(V(double(r[c]) - alpha * double(q[c])));
                }
                r[c] = V(rv);
                const double dg = diag2(k, c, i, j);
                zv = dg > 0.0 ? rv / dg : rv;
                s_z += zv;
                s_r += rv;
            }
            z[c] = V(zv);
            s_rr += rv * rv;
            s_max = fmax(s_max, fabs(rv));
            s_rz += rv * double(V(zv));
        }
        {
            double v[5] = {s_rr, s_z, s_rz, s_r, s_x};
            write_parts_max<5>(k, sync, v, s_max, red);
        }
        if (!sync()) return;
        double rz_new;
        {
            double s5[5];
            read_sums_max<5>(k, sync, s5, rmax, red);
            rr = s5[0];
            mz = proj ? s5[1] / cnt : 0.0;
            rz_new = s5[2] - mz * s5[3];
            s_r_prev = s5[3];
            s_x_prev = s5[4];
        }
        residual = l2 ? sqrt(rr) : rmax;
        if (!isfinite(residual)) { error = FLURSYS_ERR_NON_FINITE; break; }
        bool conv = l2 ? (residual <= threshold) : (residual < threshold);
        if (MIXED && (conv || ((it + 1) % in.replace_every) == 0)) {
            if (!residual_pass()) return;  // FP64 true residual replaces r
            read_residual_sums(rr, rmax, rz_new);
            residual = l2 ? sqrt(rr) : rmax;
            if (!isfinite(residual)) { error = FLURSYS_ERR_NON_FINITE; break; }
            conv = l2 ? (residual <= threshold) : (residual < threshold);
        }
        if (conv) { status = FLURSYS_LINEAR_CONVERGED; break; }
        if (fabs(rz_old) < 1.0e-30) break;
        beta = rz_new / rz_old;
        rz_old = rz_new;
        md_old = md;
        first = false;
    }
    // ---- final FP64 check ||b' - A x||_2 over fluid rows ----
    if (!sync()) return;
    double s_true = 0.0;
    for (CellIter it = first_cell(k); it.c < k.c_end; next_cell(k, it)) {
        const int c = it.c, i = it.i, j = it.j;
        if (ident(f, c)) continue;
        const double t = bval(c) - mb - apply_row<double>(k, c, i, j, x[c], [&](int m) { return x[m]; });
        s_true += t * t;
    }
    {
        double v[1] = {s_true};
        write_parts<1>(k, sync, v, red);
    }
    if (!sync()) return;
    double st1[1];
    read_sums<1>(k, sync, st1, red);
    const double true_rr = st1[0];
    if (k.lb == 0 && threadIdx.x == 0) {
        PcgResultDev *res = in.result;
        res->error = error;
        res->status = status;
        res->iterations = iterations;
        res->initial = initial;
        res->residual = residual;
        res->true_l2 = sqrt(true_rr);
        res->initial_l2 = initial_l2;
        res->device_error = in.barrier->error;
    }
}

template <typename Sync>
__device__ void sor_instance(Ctx &k, double *red, const Sync &sync) {
    const Pcg2dInstance &in = k.in;
    const uint8_t *f = in.flags;
    double *p = in.x;
    const int nx = in.nx;
    double residual = INFINITY;
    long long its = 0;
    int error = 0;
    for (long long sweep = 0; sweep < in.max_iters; ++sweep) {
        its = sweep + 1;
        for (int color = 0; color < 2; ++color) {
            for (CellIter it = first_cell(k); it.c < k.c_end; next_cell(k, it)) {
                const int c = it.c, i = it.i, j = it.j;
                if (((i + j) & 1) != color) continue;
                const uint8_t fc = f[c];
                if (fc & kCellSolid) { p[c] = 0.0; continue; }
                if (fc & kCellOutlet) { p[c] = in.outlet_pressure; continue; }
                double ap = 0.0, s = 0.0;
                if (i + 1 < nx && !solid(f, c + 1)) { ap += in.idx2; s += in.idx2 * p[c + 1]; }
                if (i > 0 && !solid(f, c - 1)) { ap += in.idx2; s += in.idx2 * p[c - 1]; }
                if (j + 1 < in.ny && !solid(f, c + nx)) { ap += in.idy2; s += in.idy2 * p[c + nx]; }
                if (j > 0 && !solid(f, c - nx)) { ap += in.idy2; s += in.idy2 * p[c - nx]; }
                if (ap > 0.0) {
                    const double old = p[c];
                    p[c] = old + in.omega * ((s - __ldg(in.rhs + c)) / ap - old);
                }
            }
            if (!sync()) return;
        }
        if (in.project && in.ref_cell >= 0) {
            const double pr = p[in.ref_cell];
            if (!sync()) return;
            for (int c = k.c_begin + threadIdx.x; c < k.c_end; c += kBlock)
                if (!solid(f, c)) p[c] -= pr;
            if (!sync()) return;
        }
        double m = 0.0;
        for (CellIter it = first_cell(k); it.c < k.c_end; next_cell(k, it)) {
            const int c = it.c, i = it.i, j = it.j;
            if (ident(f, c)) continue;
            const double p0 = p[c];
            const double pe = (i + 1 < nx && !solid(f, c + 1)) ? p[c + 1] : p0;
            const double pw = (i > 0 && !solid(f, c - 1)) ? p[c - 1] : p0;
            const double pn = (j + 1 < in.ny && !solid(f, c + nx)) ? p[c + nx] : p0;
            const double ps = (j > 0 && !solid(f, c - nx)) ? p[c - nx] : p0;
            const double lap = (pe - 2.0 * p0 + pw) * in.idx2 + (pn - 2.0 * p0 + ps) * in.idy2;
            m = fmax(m, fabs(lap - __ldg(in.rhs + c)));
        }
        write_max(k, sync, m, red);
        if (!sync()) return;
        residual = read_max(k, sync, red);
        if (!isfinite(residual)) { error = FLURSYS_ERR_NON_FINITE; break; }
        if (residual < in.tol) break;
    }
    if (k.lb == 0 && threadIdx.x == 0) {
        PcgResultDev *res = in.result;
        res->error = error;
        res->status = residual < in.tol ? FLURSYS_LINEAR_CONVERGED : FLURSYS_LINEAR_MAX_ITERATIONS;
        res->iterations = its;
        res->initial = 0.0;
        res->residual = residual;
        res->true_l2 = 0.0;
        res->initial_l2 = 0.0;
        res->device_error = in.barrier->error;
    }
}

__device__ __forceinline__ void make_ctx(Ctx &k, const Pcg2dInstance &in, int lb) {
    k.in = in;
    k.lb = lb;
    k.n = k.in.nx * k.in.ny;
    const int chunk = (k.n + k.in.nblocks - 1) / k.in.nblocks;
    k.c_begin = k.lb * chunk;
    k.c_end = k.c_begin + chunk < k.n ? k.c_begin + chunk : k.n;
    k.step_j = kBlock / k.in.nx;
    k.step_i = kBlock - k.step_j * k.in.nx;
    k.round = 0;
}

template <typename V, bool MIXED>
__global__ void __launch_bounds__(kBlock, 3) pcg2d_kernel(const Pcg2dInstance *__restrict__ insts, int ninst) {
    __shared__ double red[kRoundCols * (kBlock / 32)];
    int id = 0;
    for (int t = 0; t < ninst; ++t)
        if ((int)blockIdx.x >= insts[t].block0) id = t;
    const int lb = (int)blockIdx.x - insts[id].block0;
    if (lb >= insts[id].nblocks) return;  // spare block of the launch
    Ctx k;
    make_ctx(k, insts[id], lb);
    const GridSync sync{k.in.barrier, (unsigned)k.in.nblocks, k.in.partials, &k.in.result->device_error};
    if (k.in.solver == FLURSYS_PRESSURE_SOR) sor_instance(k, red, sync);
    else pcg_instance<V, MIXED>(k, red, sync);
}

// One instance as one thread-block cluster (grid = cluster = nblocks): the
// passes are separated by the hardware cluster barrier.
template <typename V, bool MIXED>
__global__ void __launch_bounds__(kBlock, 3) pcg2d_cluster_kernel(const Pcg2dInstance *__restrict__ inst) {
    __shared__ double red[kRoundCols * (kBlock / 32)];
    Ctx k;
    make_ctx(k, inst[0], (int)blockIdx.x);
    const ClusterSync sync{k.in.partials};
    if (k.in.solver == FLURSYS_PRESSURE_SOR) sor_instance(k, red, sync);
    else pcg_instance<V, MIXED>(k, red, sync);
}

}  // namespace

cudaError_t pcg2d_max_grid(int precision, int device, int *grid) {
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    if (precision == FLURSYS_PRECISION_MIXED)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg2d_kernel<float, true>, kBlock, 0);
    else
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg2d_kernel<double, false>, kBlock, 0);
    if (e != cudaSuccess) return e;
    *grid = sms * per_sm;
    return cudaSuccess;
}

int pcg2d_max_cluster(int precision) {
    const void *fn = precision == FLURSYS_PRECISION_MIXED ? (const void *)pcg2d_cluster_kernel<float, true>
                                                          : (const void *)pcg2d_cluster_kernel<double, false>;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return 8;  // the portable cluster size
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(16);
    cfg.blockDim = dim3(kBlock);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 16;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int size = 0;
    if (cudaOccupancyMaxPotentialClusterSize(&size, fn, &cfg) != cudaSuccess || size < 1) {
        cudaGetLastError();
        return 8;
    }
    return size;
}

cudaError_t pcg2d_launch_cluster(const Pcg2dInstance *inst_dev, int nblocks, int precision, cudaStream_t stream) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(nblocks);
    cfg.blockDim = dim3(kBlock);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = nblocks;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (precision == FLURSYS_PRECISION_MIXED) return cudaLaunchKernelEx(&cfg, pcg2d_cluster_kernel<float, true>, inst_dev);
    return cudaLaunchKernelEx(&cfg, pcg2d_cluster_kernel<double, false>, inst_dev);
}

int pcg2d_block_size() { return kBlock; }
int pcg2d_num_partials() { return kParts; }

// cudaLaunchKernelEx with the cooperative attribute: valid on a stream and
// inside stream capture (the batched solver records it in its step graph).
cudaError_t pcg2d_launch(const Pcg2dInstance *inst_dev, int ninst, int total_blocks, int precision,
                         cudaStream_t stream) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(total_blocks);
    cfg.blockDim = dim3(kBlock);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (precision == FLURSYS_PRECISION_MIXED)
        return cudaLaunchKernelEx(&cfg, pcg2d_kernel<float, true>, inst_dev, ninst);
    return cudaLaunchKernelEx(&cfg, pcg2d_kernel<double, false>, inst_dev, ninst);
}

}  // namespace flursys
