// pcg3d_seq.cu — the 3D pressure PCG as a kernel sequence in one CUDA graph.
//
// Same system, iteration order, precision modes and stop semantics as the
// persistent kernel of pcg3d.cu (see there), but each phase is its own
// high-occupancy launch and the loop runs on the device:
//
//   graph:  init -> WHILE(continue) { (dir_spmv -> update -> IF(replace) { fold -> replace }) x unroll } -> final
//
//   init      r = b - A x (FP64), sums r.r, r.z, max|r|; sets `continue`
//   dir_spmv  d = z + beta d_old formed on the fly (cells and halo), q = A d,
//             sum d.q -> alpha
//   update    x (or the FP32 increment) += alpha d, r -= alpha q, sums ->
//             stop test, beta; in MIXED mode every `replace_every`
//             iterations and before accepting convergence it raises `replace`
//   fold      x += increment (MIXED)
//   replace   r = b - A x in FP64 (residual replacement), sums -> stop test, beta
//   final     FP64 ||b - A x||_2 of the returned pressure
//
// Reductions use the last-block pattern: every block writes one partial,
// fences, and bumps a counter; the block that arrives last sums the partials
// in block order (deterministic) and updates the scalar state, which later
// launches read. Nothing spins. The stencil launches walk one tile each
// (32 x 8 columns, a chunk of planes) with the 2.5D scheme of pcg3d.cu; the
// hardware schedules tiles dynamically across the SMs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <type_traits>

#include "common.cuh"
#include "pcg3d.cuh"
#include "pcg3d_seq.cuh"
#include "pcg3d_res.cuh"
#include "tma.cuh"

namespace flursys {

namespace {

constexpr int TX = 32;
constexpr int TY = 8;
constexpr int kBlock = TX * TY;

struct SeqGeo {
    int nx, ny, nz, nxy, n;
    int tiles_x, tiles_y, kc, chunks;  // tile / direct sweeps: 32 x 8 columns
    int tiles_yw, kcw, chunksw;        // warp sweep: 32 x (8 * kRyOperand) columns
    int tiles_xv, tiles_yv, kcv, chunksv;  // vector sweep: (32 W) x (8 kRyVec) columns
    int kcp, chunksp;                      // staged sweep: the vector sweep's columns, longer chunks
    double ix2, iy2, iz2;
    double inv_diag[27];  // 1/diag by missing-neighbour class 9*mx + 3*my + mz
};

struct SeqArgs {
    SeqGeo g;
    double *x;
    const double *rhs;
    void *r, *d0, *d1, *q;
    float *dx;
    double *partials;  // nblocks * kSlots
    CgSeqState *st;
    const unsigned char *row_class;
    cudaGraphConditionalHandle h_loop, h_replace;
    int stop_rule;
    double tol, atol, rtol;
    long long max_iters;
    int replace_every;
    int nblocks_stencil, nblocks_point;
    int graph;   // 1: kernels run inside the solve graph and set its conditionals
    int sweep;   // stencil scheme of the operand pass (kSweep*)
    int nblocks_dir;  // grid of the operand pass
    // single-reduction variant (MIXED): buffer sets 0/1 of r and p alternate
    // per iteration; dx is updated in place
    float *cr[2], *cp[2];
    int cg1;          // 1: single-reduction variant
    int cg1_tz;       // planes per tile of its step kernel (4 or 8)
    int nblocks_cg1;  // grid of its step kernel
};

enum SweepKind : int { kSweepWarp = 0, kSweepTile = 1, kSweepDirect = 2, kSweepVec = 3, kSweepPipe = 4 };
constexpr int kRyVec = 2;  // rows per lane of the vectorised operand pass
constexpr int kRyOperand = 4;  // rows per lane of the warp sweep (FP32; half of it in FP64)

__device__ __forceinline__ void set_cond(const SeqArgs &a, cudaGraphConditionalHandle h, unsigned v) {
    if (a.graph) cudaGraphSetConditional(h, v);
}

__device__ __forceinline__ int miss(int i, int n) { return (i == 0) + (i == n - 1); }

constexpr int kSlots = 8;  // partial-sum slots per block

// Writes this block's NS sums (slots 0..NS-1) and, with MAX, the block
// maximum of mx (slot NS); returns true in the block that arrives last.
template <int NS, bool MAX>
__device__ __forceinline__ bool arrive_n(double (&v)[NS], double mx, double *partials, unsigned *counter,
                                         double *red) {
    __shared__ bool s_last;
    const int nb = gridDim.x;
    block_reduce_n<kBlock, NS, MAX>(v, mx, red);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NS; ++k) partials[blockIdx.x * kSlots + k] = v[k];
        if (MAX) partials[blockIdx.x * kSlots + NS] = mx;
        __threadfence();
        const unsigned prev = atomicAdd(counter, 1u);
        s_last = prev == (unsigned)nb - 1u;
    }
    __syncthreads();
    if (s_last) __threadfence();
    return s_last;
}

// Fixed-order sums (and maximum) over all blocks' partials.
template <int NS, bool MAX>
__device__ __forceinline__ void finish_n(double (&out)[NS], double &mx, const double *partials, double *red) {
    const int nb = gridDim.x;
#pragma unroll
    for (int k = 0; k < NS; ++k) out[k] = 0.0;
    mx = 0.0;
    for (int b = threadIdx.x; b < nb; b += kBlock) {
#pragma unroll
        for (int k = 0; k < NS; ++k) out[k] += __ldcg(partials + b * kSlots + k);
        if (MAX) mx = fmax(mx, __ldcg(partials + b * kSlots + NS));
    }
    block_reduce_n<kBlock, NS, MAX>(out, mx, red);
}

// NV = 1: one sum. NV = 3: sums in slots 0 and 1, a maximum in slot 2.
template <int NV>
__device__ __forceinline__ bool reduce_arrive(const double (&v)[NV], double *partials, unsigned *counter,
                                              double *red) {
    static_assert(NV == 1 || NV == 3, "one sum, or two sums and a maximum");
    if (NV == 1) {
        double t[1] = {v[0]};
        return arrive_n<1, false>(t, 0.0, partials, counter, red);
    }
    double t[2] = {v[0], v[NV > 1 ? 1 : 0]};
    return arrive_n<2, true>(t, v[NV > 2 ? 2 : 0], partials, counter, red);
}

template <int NV>
__device__ __forceinline__ void reduce_finish(double (&out)[NV], const double *partials, double *red) {
    static_assert(NV == 1 || NV == 3, "one sum, or two sums and a maximum");
    double mx;
    if (NV == 1) {
        double t[1];
        finish_n<1, false>(t, mx, partials, red);
        out[0] = t[0];
        return;
    }
    double t[2];
    finish_n<2, true>(t, mx, partials, red);
    out[0] = t[0];
    out[NV > 1 ? 1 : 0] = t[1];
    out[NV > 2 ? 2 : 0] = mx;
}

// One tile of the 2.5D sweep (see pcg3d.cu). Raw inputs are prefetched two
// planes ahead for the column and the x/y halo.
template <typename Load, typename Make, typename Emit>
__device__ __forceinline__ void tile_sweep(const SeqGeo &g, int t, void *tile_mem, Load load, Make make, Emit emit) {
    using Raw = decltype(load(0));
    using T = decltype(make(load(0), 0, false));
    constexpr int SW = TX + 2;
    const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
    const T wx = T(g.ix2), wy = T(g.iy2), wz = T(g.iz2);
    T *ts = reinterpret_cast<T *>(tile_mem);
    const int h = threadIdx.x;
    const bool halo_thread = h < 2 * TX + 2 * TY;
    const int ch = t % g.chunks, col = t / g.chunks;
    const int i0 = (col % g.tiles_x) * TX, j0 = (col / g.tiles_x) * TY;
    const int k0 = ch * g.kc, k1 = min(g.nz, k0 + g.kc);
    const int kmax = min(k1, g.nz - 1);
    const int i = i0 + tx, j = j0 + ty;
    const bool in = i < g.nx && j < g.ny;
    const int base = in ? j * g.nx + i : 0;
    const int cxy = 9 * miss(i, g.nx) + 3 * miss(j, g.ny);
    const T wxm = (in && i > 0) ? wx : T(0), wxp = (in && i + 1 < g.nx) ? wx : T(0);
    const T wym = (in && j > 0) ? wy : T(0), wyp = (in && j + 1 < g.ny) ? wy : T(0);
    const T dgxy = wxm + wxp + wym + wyp;
    const bool pcol = in && base == 0;
    int hi = 0, hj = 0;
    if (h < TX) { hi = i0 + h; hj = j0 - 1; }
    else if (h < 2 * TX) { hi = i0 + h - TX; hj = j0 + TY; }
    else if (h < 2 * TX + TY) { hi = i0 - 1; hj = j0 + h - 2 * TX; }
    else { hi = i0 + TX; hj = j0 + h - 2 * TX - TY; }
    const bool hv = halo_thread && hi >= 0 && hi < g.nx && hj >= 0 && hj < g.ny;
    const int hbase = hv ? hj * g.nx + hi : 0;
    const int hcls = hv ? 9 * miss(hi, g.nx) + 3 * miss(hj, g.ny) : 0;
    const int hslot = halo_thread ? (hj - j0 + 1) * SW + (hi - i0 + 1) : 0;
    const bool hpcol = hv && hbase == 0;
    T below = T(0), cur = T(0);
    Raw a1{}, a2{}, h1{}, h2{};
    if (in) {
        if (k0 > 0) below = make(load(base + (k0 - 1) * g.nxy), cxy + miss(k0 - 1, g.nz), false);
        cur = make(load(base + k0 * g.nxy), cxy + miss(k0, g.nz), pcol && k0 == 0);
        if (k0 + 1 <= kmax) a1 = load(base + (k0 + 1) * g.nxy);
        if (k0 + 2 <= kmax) a2 = load(base + (k0 + 2) * g.nxy);
    }
    if (hv) {
        h1 = load(hbase + k0 * g.nxy);
        if (k0 + 1 < k1) h2 = load(hbase + (k0 + 1) * g.nxy);
    }
    for (int k = k0; k < k1; ++k) {
        const int mk = miss(k, g.nz);
        T above = T(0);
        if (in) {
            if (k + 1 < g.nz) above = make(a1, cxy + miss(k + 1, g.nz), false);
            a1 = a2;
            if (k + 3 <= kmax) a2 = load(base + (k + 3) * g.nxy);
        }
        T hval = T(0);
        if (hv) {
            hval = make(h1, hcls + mk, hpcol && k == 0);
            h1 = h2;
            if (k + 2 < k1) h2 = load(hbase + (k + 2) * g.nxy);
        }
        const int sp = (ty + 1) * SW + tx + 1;
        ts[sp] = cur;
        if (halo_thread) ts[hslot] = hval;
        __syncthreads();
        if (in) {
            const T wzm = k > 0 ? wz : T(0), wzp = k + 1 < g.nz ? wz : T(0);
            const T ax = (dgxy + wzm + wzp) * cur -
                         (wxm * ts[sp - 1] + wxp * ts[sp + 1] + wym * ts[sp - SW] + wyp * ts[sp + SW] +
                          wzm * below + wzp * above);
            const bool pin = pcol && k == 0;
            emit(base + k * g.nxy, cxy + mk, pin, cur, pin ? cur : ax);
        }
        __syncthreads();
        below = cur;
        cur = above;
    }
}

// Alternative sweep without shared memory: each thread marches its column
// through the chunk with the planes below/above in registers and reads its
// four in-plane neighbours' raw inputs directly (L1-cached), forming their
// operand values itself. No block barrier.
template <typename Load, typename Make, typename Emit>
__device__ __forceinline__ void direct_sweep(const SeqGeo &g, int t, Load load, Make make, Emit emit) {
    using Raw = decltype(load(0));
    using T = decltype(make(load(0), 0, false));
    const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
    const T wx = T(g.ix2), wy = T(g.iy2), wz = T(g.iz2);
    const int ch = t % g.chunks, col = t / g.chunks;
    const int i0 = (col % g.tiles_x) * TX, j0 = (col / g.tiles_x) * TY;
    const int k0 = ch * g.kc, k1 = min(g.nz, k0 + g.kc);
    const int kmax = min(k1, g.nz - 1);
    const int i = i0 + tx, j = j0 + ty;
    if (i >= g.nx || j >= g.ny) return;
    const int base = j * g.nx + i;
    const int mi = miss(i, g.nx), mj = miss(j, g.ny);
    const int cxy = 9 * mi + 3 * mj;
    const bool hw = i > 0, he = i + 1 < g.nx, hs = j > 0, hn = j + 1 < g.ny;
    const T wxm = hw ? wx : T(0), wxp = he ? wx : T(0), wym = hs ? wy : T(0), wyp = hn ? wy : T(0);
    // classes of the in-plane neighbours (their own missing counts)
    const int cw = 9 * miss(i - 1, g.nx) + 3 * mj, ce = 9 * miss(i + 1, g.nx) + 3 * mj;
    const int cs = 9 * mi + 3 * miss(j - 1, g.ny), cn = 9 * mi + 3 * miss(j + 1, g.ny);
    const bool pcol = base == 0;
    T below = T(0), cur = T(0);
    Raw a1{}, a2{};
    if (k0 > 0) below = make(load(base + (k0 - 1) * g.nxy), cxy + miss(k0 - 1, g.nz), false);
    cur = make(load(base + k0 * g.nxy), cxy + miss(k0, g.nz), pcol && k0 == 0);
    if (k0 + 1 <= kmax) a1 = load(base + (k0 + 1) * g.nxy);
    if (k0 + 2 <= kmax) a2 = load(base + (k0 + 2) * g.nxy);
    for (int k = k0; k < k1; ++k) {
        const int mk = miss(k, g.nz);
        const int c = base + k * g.nxy;
        const Raw rw = hw ? load(c - 1) : Raw{}, re = he ? load(c + 1) : Raw{};
        const Raw rs = hs ? load(c - g.nx) : Raw{}, rn = hn ? load(c + g.nx) : Raw{};
        T above = T(0);
        if (k + 1 < g.nz) above = make(a1, cxy + miss(k + 1, g.nz), false);
        a1 = a2;
        if (k + 3 <= kmax) a2 = load(base + (k + 3) * g.nxy);
        const bool k0p = k == 0;
        const T vw = hw ? make(rw, cw + mk, k0p && c - 1 == 0) : T(0);
        const T ve = he ? make(re, ce + mk, false) : T(0);
        const T vs = hs ? make(rs, cs + mk, k0p && c - g.nx == 0) : T(0);
        const T vn = hn ? make(rn, cn + mk, false) : T(0);
        const T wzm = k > 0 ? wz : T(0), wzp = k + 1 < g.nz ? wz : T(0);
        const T ax = (wxm + wxp + wym + wyp + wzm + wzp) * cur -
                     (wxm * vw + wxp * ve + wym * vs + wyp * vn + wzm * below + wzp * above);
        const bool pin = pcol && k0p;
        emit(c, cxy + mk, pin, cur, pin ? cur : ax);
        below = cur;
        cur = above;
    }
}

// Barrier-free sweep: warp w of the block owns rows [jw, jw + RY) of a
// 32-column tile; lane l owns column i0 + l of those rows and marches them
// through the chunk of planes. In-plane neighbours come from the lane's own
// rows (y), from two halo rows it loads itself (y), and from the adjacent
// lanes by shuffle (x; lanes 0 and 31 load the tile's x halo). The planes
// below and above stay in registers; raw inputs are prefetched two planes
// ahead. A block covers 32 x (8 RY) columns.
template <int RY, typename Load, typename Make, typename Emit>
__device__ __forceinline__ void warp_sweep(const SeqGeo &g, int t, Load load, Make make, Emit emit) {
    using Raw = decltype(load(0));
    using T = decltype(make(load(0), 0, false));
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const T wx = T(g.ix2), wy = T(g.iy2), wz = T(g.iz2);
    const int ch = t % g.chunksw, col = t / g.chunksw;
    const int i0 = (col % g.tiles_x) * TX;
    const int jw = (col / g.tiles_x) * (TY * RY) + w * RY;
    if (jw >= g.ny) return;  // whole warp idle (uniform)
    const int k0 = ch * g.kcw, k1 = min(g.nz, k0 + g.kcw);
    const int kmax = min(k1, g.nz - 1);
    const int i = i0 + lane;
    const bool inx = i < g.nx;
    const int ic = inx ? i : g.nx - 1;  // clamped column for address math of idle lanes
    const int mi = miss(ic, g.nx);
    const T wxm = (inx && i > 0) ? wx : T(0), wxp = (inx && i + 1 < g.nx) ? wx : T(0);
    // rows of this warp: jw .. jw + RY - 1 (row m valid if jw + m < ny)
    // halo loads: lane 0 the west column, lane 31 the east column (own rows)
    const bool xw = lane == 0 && i0 > 0, xe = lane == 31 && i0 + TX < g.nx;
    const int xcol = xw ? i0 - 1 : (xe ? i0 + TX : ic);
    const int mxc = miss(xcol, g.nx);
    const bool ys = jw > 0, yn = jw + RY < g.ny;  // south / north halo rows exist
    T below[RY], cur[RY];
    Raw a1[RY], a2[RY];
    auto rowok = [&](int m) { return jw + m < g.ny; };
    auto cell = [&](int col_i, int row, int k) { return (k * g.ny + row) * g.nx + col_i; };
#pragma unroll
    for (int m = 0; m < RY; ++m) {
        below[m] = T(0);
        cur[m] = T(0);
        a1[m] = Raw{};
        a2[m] = Raw{};
        if (rowok(m)) {
            const int row = jw + m, cls = 9 * mi + 3 * miss(row, g.ny);
            if (k0 > 0) below[m] = make(load(cell(ic, row, k0 - 1)), cls + miss(k0 - 1, g.nz), false);
            cur[m] = make(load(cell(ic, row, k0)), cls + miss(k0, g.nz), cell(ic, row, k0) == 0);
            if (k0 + 1 <= kmax) a1[m] = load(cell(ic, row, k0 + 1));
            if (k0 + 2 <= kmax) a2[m] = load(cell(ic, row, k0 + 2));
        }
    }
    for (int k = k0; k < k1; ++k) {
        const int mk = miss(k, g.nz);
        // in-plane halo raw inputs of plane k (L1/L2 hits: neighbours' data)
        const Raw rs = ys ? load(cell(ic, jw - 1, k)) : Raw{};
        const Raw rn = yn ? load(cell(ic, jw + RY, k)) : Raw{};
        Raw rx[RY];
#pragma unroll
        for (int m = 0; m < RY; ++m) rx[m] = ((xw || xe) && rowok(m)) ? load(cell(xcol, jw + m, k)) : Raw{};
        T above[RY];
#pragma unroll
        for (int m = 0; m < RY; ++m) {
            above[m] = T(0);
            if (rowok(m)) {
                if (k + 1 < g.nz) above[m] = make(a1[m], 9 * mi + 3 * miss(jw + m, g.ny) + miss(k + 1, g.nz), false);
                a1[m] = a2[m];
                if (k + 3 <= kmax) a2[m] = load(cell(ic, jw + m, k + 3));
            }
        }
        const T vs = ys ? make(rs, 9 * mi + 3 * miss(jw - 1, g.ny) + mk, cell(ic, jw - 1, k) == 0) : T(0);
        const T vn = yn ? make(rn, 9 * mi + 3 * miss(jw + RY, g.ny) + mk, false) : T(0);
        const T wzm = k > 0 ? wz : T(0), wzp = k + 1 < g.nz ? wz : T(0);
#pragma unroll
        for (int m = 0; m < RY; ++m) {
            // x neighbours by shuffle; the tile edges take the loaded halo
            const T xh = ((xw || xe) && rowok(m)) ? make(rx[m], 9 * mxc + 3 * miss(jw + m, g.ny) + mk,
                                                          cell(xcol, jw + m, k) == 0)
                                                   : T(0);
            T west = __shfl_up_sync(0xffffffffu, cur[m], 1);
            T east = __shfl_down_sync(0xffffffffu, cur[m], 1);
            if (lane == 0) west = xh;
            if (lane == 31) east = xh;
            const int row = jw + m;
            if (inx && rowok(m)) {
                const T south = m > 0 ? cur[m > 0 ? m - 1 : 0] : vs;
                const T north = m + 1 < RY ? cur[m + 1 < RY ? m + 1 : 0] : vn;
                const T wym = row > 0 ? wy : T(0), wyp = row + 1 < g.ny ? wy : T(0);
                const T ax = (wxm + wxp + wym + wyp + wzm + wzp) * cur[m] -
                             (wxm * west + wxp * east + wym * south + wyp * north + wzm * below[m] +
                              wzp * above[m]);
                const int c = cell(i, row, k);
                const bool pin = c == 0;
                emit(c, 9 * mi + 3 * miss(row, g.ny) + mk, pin, cur[m], pin ? cur[m] : ax);
            }
        }
#pragma unroll
        for (int m = 0; m < RY; ++m) {
            below[m] = cur[m];
            cur[m] = above[m];
        }
    }
}

__device__ __forceinline__ bool stop_ok(const SeqArgs &a, double res, double thr) {
    return a.stop_rule == FLURSYS_STOP_REL_L2 ? res <= thr : res < thr;
}

// Residual r = b - A x (FP64) over one tile with its sums; shared by init and replace.
template <typename V, bool MIXED>
__device__ __forceinline__ void residual_tile(const SeqArgs &a, V *r, void *tile, double &srr, double &srz,
                                              double &smax, bool zero_dx) {
    const SeqGeo &g = a.g;
    tile_sweep(
        g, blockIdx.x, tile, [&](int c) -> double { return a.x[c]; },
        [&](double v, int, bool pin) -> double { return pin ? 0.0 : v; },
        [&](int c, int cls, bool pin, double, double ax) {
            const double rr = pin ? 0.0 : -__ldg(a.rhs + c) - ax;
            const V rv = V(rr);
            r[c] = rv;
            if (MIXED && zero_dx) a.dx[c] = 0.f;
            const double rd = double(rv);
            srr += rd * rd;
            srz += rd * rd * (pin ? 1.0 : g.inv_diag[cls]);
            smax = fmax(smax, fabs(rd));
        });
}

template <typename V, bool MIXED>
__global__ void __launch_bounds__(kBlock) seq_init(SeqArgs a) {
    __shared__ double tile[(TY + 2) * (TX + 2)];
    __shared__ double red[kSlots * (kBlock / 32)];
    double srr = 0.0, srz = 0.0, smax = 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) a.x[0] = 0.0;
    residual_tile<V, MIXED>(a, static_cast<V *>(a.r), tile, srr, srz, smax, true);
    const double v[3] = {srr, srz, smax};
    if (!reduce_arrive<3>(v, a.partials, &a.st->counter, red)) return;
    double o[3];
    reduce_finish<3>(o, a.partials, red);
    if (threadIdx.x == 0) {
        CgSeqState *s = a.st;
        const bool l2 = a.stop_rule == FLURSYS_STOP_REL_L2;
        s->counter = 0;
        s->initial_l2 = sqrt(o[0]);
        s->initial = l2 ? s->initial_l2 : o[2];
        s->threshold = l2 ? a.atol + a.rtol * s->initial : a.tol;
        s->residual = s->initial;
        s->rz_old = o[1];
        s->beta = 0.0;
        s->first = 1;
        s->iterations = 0;
        s->error = 0;
        s->replace = 0;
        s->pending_conv = 0;
        const bool done = stop_ok(a, s->initial, s->threshold);
        s->status = done ? FLURSYS_LINEAR_CONVERGED : FLURSYS_LINEAR_MAX_ITERATIONS;
        s->done = done || a.max_iters <= 0;
        set_cond(a, a.h_loop, s->done ? 0u : 1u);
    }
}

template <typename V, bool MIXED>
__global__ void __launch_bounds__(kBlock) seq_dir_spmv(SeqArgs a) {
    __shared__ double tile[(TY + 2) * (TX + 2)];
    __shared__ double red[kSlots * (kBlock / 32)];
    const CgSeqState *s = a.st;
    if (s->done) return;  // the solve has finished (host-driven mode, or a later iteration of an unrolled body)
    const double beta = s->beta;
    const bool first = s->first != 0;
    const int parity = (int)(s->iterations & 1);  // d buffers alternate per iteration
    V *r = static_cast<V *>(a.r);
    V *dcur = static_cast<V *>(parity ? a.d1 : a.d0);
    const V *dold = static_cast<const V *>(parity ? a.d0 : a.d1);
    V *q = static_cast<V *>(a.q);
    const SeqGeo &g = a.g;
    const V vbeta = V(beta);
    struct RawA {
        V r, d;
    };
    double sdq = 0.0;
    auto load_a = [&](int c) -> RawA { return RawA{r[c], first ? V(0) : dold[c]}; };
    auto make_a = [&](RawA v, int cls, bool pin) -> V {
        if (pin) return V(0);
        const V z = V(double(v.r) * g.inv_diag[cls]);
        return first ? z : V(z + vbeta * v.d);
    };
    auto emit_a = [&](int c, int, bool, V dc, V qc) {
        dcur[c] = dc;
        q[c] = qc;
        sdq += double(dc) * double(qc);
    };
    if (a.sweep == kSweepWarp) warp_sweep<(sizeof(V) == 4 ? kRyOperand : kRyOperand / 2)>(g, blockIdx.x, load_a, make_a, emit_a);
    else if (a.sweep == kSweepDirect) direct_sweep(g, blockIdx.x, load_a, make_a, emit_a);
    else tile_sweep(g, blockIdx.x, tile, load_a, make_a, emit_a);
    const double v[1] = {sdq};
    if (!reduce_arrive<1>(v, a.partials, &a.st->counter, red)) return;
    double o[1];
    reduce_finish<1>(o, a.partials, red);
    if (threadIdx.x == 0) {
        CgSeqState *w = a.st;
        w->counter = 0;
        const double dq = o[0];
        if (fabs(dq) < 1.0e-30 || !isfinite(dq) || !isfinite(w->rz_old / dq)) {
            w->error = FLURSYS_ERR_BREAKDOWN;
            w->done = 1;
            w->alpha = 0.0;
        } else {
            w->alpha = w->rz_old / dq;
        }
    }
}

// ---------------------------------------------------------------------------
// Vectorised operand pass (the hot kernel): d = z + beta d_old, q = A d, d.q.
// Warp w of a block owns rows [row0, row0 + RY) of a strip of 32*W columns;
// lane l owns the W consecutive cells [i0 + W l, i0 + W l + W) of each row
// (one float4 / double2 load per array per row). x neighbours: inside the
// lane's vector, then the adjacent lanes by shuffle, and at the strip edges a
// scalar halo loaded by lanes 0 and 31. y neighbours: the lane's own rows
// plus one halo row below and above (prefetched with the rows). z
// neighbours: registers, raw inputs prefetched one plane ahead. No shared
// memory tiles and no block barriers in the plane loop.
// Requires nx % W == 0 (checked on the host; the tile sweep serves the rest).
// ---------------------------------------------------------------------------
template <typename V>
struct VecOf;
template <>
struct VecOf<float> {
    using T = float4;
    static constexpr int W = 4;
};
template <>
struct VecOf<double> {
    using T = double2;
    static constexpr int W = 2;
};

template <typename V, bool MIXED, int RY>
__global__ void __launch_bounds__(kBlock, 2) seq_dir_vec(SeqArgs a) {
    using VT = typename VecOf<V>::T;
    constexpr int W = VecOf<V>::W;
    constexpr int XW = 32 * W;
    __shared__ double red[kSlots * (kBlock / 32)];
    __shared__ V idg[27];
    const SeqGeo &g = a.g;
    if (threadIdx.x < 27) idg[threadIdx.x] = V(g.inv_diag[threadIdx.x]);
    __syncthreads();
    const CgSeqState *s = a.st;
    if (s->done) return;  // the solve has finished (host-driven mode, or a later iteration of an unrolled body)
    const bool first = s->first != 0;
    const V beta = V(s->beta);
    const int parity = (int)(s->iterations & 1);
    const V *r = static_cast<const V *>(a.r);
    V *dcur = static_cast<V *>(parity ? a.d1 : a.d0);
    const V *dold = static_cast<const V *>(parity ? a.d0 : a.d1);
    V *q = static_cast<V *>(a.q);
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int t = blockIdx.x;
    const int ch = t % g.chunksv, col = t / g.chunksv;
    const int i0 = (col % g.tiles_xv) * XW;
    const int row0 = (col / g.tiles_xv) * (TY * RY) + wp * RY;
    double sdq = 0.0;
    if (row0 < g.ny) {
        const int k0 = ch * g.kcv, k1 = min(g.nz, k0 + g.kcv);
        const int ib = i0 + lane * W;
        const bool inx = ib < g.nx;
        const int ibc = inx ? ib : g.nx - W;  // idle lanes read a valid vector
        const V wx = V(g.ix2), wy = V(g.iy2), wz = V(g.iz2);
        // x weights of the lane's first and last element (domain walls)
        const V wxm0 = (inx && ib > 0) ? wx : V(0);
        const V wxpL = (inx && ib + W < g.nx) ? wx : V(0);
        const int mx0 = miss(ibc, g.nx), mxL = miss(ibc + W - 1, g.nx);
        const bool hw = lane == 0 && i0 > 0, he = lane == 31 && i0 + XW < g.nx;
        const int xh = hw ? i0 - 1 : (he ? i0 + XW : 0);
        const int mxh = miss(xh, g.nx);
        const bool ys = row0 > 0, yn = row0 + RY < g.ny;
        auto ld = [&](const V *p, int c) -> VT { return *reinterpret_cast<const VT *>(p + c); };
        auto el = [](const VT &v, int e) -> V { return reinterpret_cast<const V *>(&v)[e]; };
        auto idx = [&](int i, int row, int k) { return (k * g.ny + row) * g.nx + i; };
        // d_new of W cells of one row from raw r and d_old vectors
        auto make = [&](const VT &rv, const VT &dv, int row, int k, V (&out)[W]) {
            const int cyz = 3 * miss(row, g.ny) + miss(k, g.nz);
            const V mid = idg[cyz];
#pragma unroll
            for (int e = 0; e < W; ++e) {
                V id = mid;
                if (e == 0 && mx0) id = idg[9 * mx0 + cyz];
                if (e == W - 1 && mxL) id = idg[9 * mxL + cyz];
                const V z = el(rv, e) * id;
                out[e] = first ? z : V(z + beta * el(dv, e));
            }
            if (k == 0 && row == 0 && ibc == 0) out[0] = V(0);  // pinned cell
        };
        auto make1 = [&](V rv, V dv, int i, int row, int k) -> V {
            if (k == 0 && row == 0 && i == 0) return V(0);
            const V z = rv * idg[9 * miss(i, g.nx) + 3 * miss(row, g.ny) + miss(k, g.nz)];
            return first ? z : V(z + beta * dv);
        };
        V below[RY][W], cur[RY][W], above[RY][W];
        VT nr[RY], nd[RY];        // raw inputs of the next plane (own rows)
        VT sr, sd, hr, hd;        // raw inputs of the y halo rows of the next plane
        V xr[RY], xd[RY];         // x halo scalars of the next plane
        const VT zero{};
        auto load_plane = [&](int k) {
#pragma unroll
            for (int m = 0; m < RY; ++m) {
                const int row = row0 + m;
                if (row < g.ny) {
                    const int c = idx(ibc, row, k);
                    nr[m] = ld(r, c);
                    nd[m] = first ? zero : ld(dold, c);
                    if (hw || he) {
                        const int cx = idx(xh, row, k);
                        xr[m] = r[cx];
                        xd[m] = first ? V(0) : dold[cx];
                    }
                }
            }
            if (ys) { const int c = idx(ibc, row0 - 1, k); sr = ld(r, c); sd = first ? zero : ld(dold, c); }
            if (yn) { const int c = idx(ibc, row0 + RY, k); hr = ld(r, c); hd = first ? zero : ld(dold, c); }
        };
        // prologue: planes k0-1 (below), k0 (cur); raw k0+1 in flight
#pragma unroll
        for (int m = 0; m < RY; ++m)
#pragma unroll
            for (int e = 0; e < W; ++e) below[m][e] = cur[m][e] = above[m][e] = V(0);
        V vs[W], vn[W], vxh[RY];
        if (k0 > 0) {
            load_plane(k0 - 1);
#pragma unroll
            for (int m = 0; m < RY; ++m)
                if (row0 + m < g.ny) make(nr[m], nd[m], row0 + m, k0 - 1, below[m]);
        }
        load_plane(k0);
#pragma unroll
        for (int m = 0; m < RY; ++m)
            if (row0 + m < g.ny) make(nr[m], nd[m], row0 + m, k0, cur[m]);
#pragma unroll
        for (int e = 0; e < W; ++e) { vs[e] = V(0); vn[e] = V(0); }
        if (ys) make(sr, sd, row0 - 1, k0, vs);
        if (yn) make(hr, hd, row0 + RY, k0, vn);
#pragma unroll
        for (int m = 0; m < RY; ++m) vxh[m] = (hw || he) && row0 + m < g.ny ? make1(xr[m], xd[m], xh, row0 + m, k0) : V(0);
        if (k0 + 1 < g.nz) load_plane(k0 + 1);
        for (int k = k0; k < k1; ++k) {
            // operand of plane k+1 for the own rows (its raw inputs landed during plane k-1)
            const bool has_above = k + 1 < g.nz;
            V vs1[W], vn1[W], vxh1[RY];
#pragma unroll
            for (int e = 0; e < W; ++e) { vs1[e] = V(0); vn1[e] = V(0); }
            if (has_above) {
#pragma unroll
                for (int m = 0; m < RY; ++m)
                    if (row0 + m < g.ny) make(nr[m], nd[m], row0 + m, k + 1, above[m]);
                if (ys) make(sr, sd, row0 - 1, k + 1, vs1);
                if (yn) make(hr, hd, row0 + RY, k + 1, vn1);
#pragma unroll
                for (int m = 0; m < RY; ++m)
                    vxh1[m] = (hw || he) && row0 + m < g.ny ? make1(xr[m], xd[m], xh, row0 + m, k + 1) : V(0);
            } else {
#pragma unroll
                for (int m = 0; m < RY; ++m) {
                    vxh1[m] = V(0);
#pragma unroll
                    for (int e = 0; e < W; ++e) above[m][e] = V(0);
                }
            }
            if (k + 2 < g.nz && k + 2 <= k1) load_plane(k + 2);  // next plane's loads in flight
            const V wzm = k > 0 ? wz : V(0), wzp = has_above ? wz : V(0);
#pragma unroll
            for (int m = 0; m < RY; ++m) {
                const int row = row0 + m;
                // shuffles are warp-uniform: every lane takes part
                V west = __shfl_up_sync(0xffffffffu, cur[m][W - 1], 1);
                V east = __shfl_down_sync(0xffffffffu, cur[m][0], 1);
                if (lane == 0) west = hw ? vxh[m] : V(0);
                if (lane == 31) east = he ? vxh[m] : V(0);
                if (!inx || row >= g.ny) continue;
                const V wym = row > 0 ? wy : V(0), wyp = row + 1 < g.ny ? wy : V(0);
                V dv[W], qv[W];
#pragma unroll
                for (int e = 0; e < W; ++e) {
                    const V wxm = e == 0 ? wxm0 : wx, wxp = e == W - 1 ? wxpL : wx;
                    const V xm = e == 0 ? west : cur[m][e - 1 < 0 ? 0 : e - 1];
                    const V xp = e == W - 1 ? east : cur[m][e + 1 < W ? e + 1 : W - 1];
                    const V ysv = m > 0 ? cur[m > 0 ? m - 1 : 0][e] : vs[e];
                    const V ynv = m + 1 < RY ? cur[m + 1 < RY ? m + 1 : 0][e] : vn[e];
                    const V c0 = cur[m][e];
                    V ax = (wxm + wxp + wym + wyp + wzm + wzp) * c0 -
                           (wxm * xm + wxp * xp + wym * ysv + wyp * ynv + wzm * below[m][e] + wzp * above[m][e]);
                    if (k == 0 && row == 0 && ib + e == 0) ax = c0;  // identity row of the pinned cell
                    dv[e] = c0;
                    qv[e] = ax;
                    sdq += double(c0) * double(ax);
                }
                const int c = idx(ib, row, k);
                *reinterpret_cast<VT *>(dcur + c) = *reinterpret_cast<const VT *>(dv);
                *reinterpret_cast<VT *>(q + c) = *reinterpret_cast<const VT *>(qv);
            }
#pragma unroll
            for (int m = 0; m < RY; ++m) {
                vxh[m] = vxh1[m];
#pragma unroll
                for (int e = 0; e < W; ++e) {
                    below[m][e] = cur[m][e];
                    cur[m][e] = above[m][e];
                }
            }
#pragma unroll
            for (int e = 0; e < W; ++e) { vs[e] = vs1[e]; vn[e] = vn1[e]; }
        }
    }
    const double v[1] = {sdq};
    if (!reduce_arrive<1>(v, a.partials, &a.st->counter, red)) return;
    double o[1];
    reduce_finish<1>(o, a.partials, red);
    if (threadIdx.x == 0) {
        CgSeqState *w = a.st;
        w->counter = 0;
        const double dq = o[0];
        if (fabs(dq) < 1.0e-30 || !isfinite(dq) || !isfinite(w->rz_old / dq)) {
            w->error = FLURSYS_ERR_BREAKDOWN;
            w->done = 1;
            w->alpha = 0.0;
        } else {
            w->alpha = w->rz_old / dq;
        }
    }
}

// ---------------------------------------------------------------------------
// seq_dir_pipe: the MIXED operand pass with its raw inputs staged through
// shared memory by cp.async. A block owns the vector sweep's column tile
// (128 cells of x by 16 rows) and marches a long chunk of planes; while
// plane k is computed, the raw r and d_old of planes k+2 and k+3 are in
// flight (a ring of kPipeSlots planes: the tile's 16 rows, the two y-halo
// rows and the two x-halo columns), so the latency of the loads is hidden
// by a whole plane of work and no register holds data in flight. The
// arithmetic is that of seq_dir_vec: d = z + beta d_old formed for the
// cells and their neighbours, q = A d with x neighbours by warp shuffle,
// d.q accumulated in FP64; cells outside the grid are staged as zeros.
// ---------------------------------------------------------------------------
constexpr int kPipeX = 128, kPipeY = 16, kPipeSlots = 5;
constexpr int kPipeRows = kPipeY + 2;                        // rows -1 .. 16
constexpr int kPipeArr = kPipeRows * kPipeX + 2 * kPipeY;    // floats per array per slot (+ x halos)
constexpr int kPipeSmem = kPipeSlots * 2 * kPipeArr * 4;      // bytes

__device__ __forceinline__ void cp_async16(void *dst, const void *src, bool valid) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src, bool valid) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(valid ? 4 : 0) : "memory");
}

__global__ void __launch_bounds__(kBlock, 2) seq_dir_pipe(SeqArgs a) {
    extern __shared__ __align__(16) float pipe_smem[];
    __shared__ double red[kSlots * (kBlock / 32)];
    __shared__ float idg[27];
    const SeqGeo &g = a.g;
    if (threadIdx.x < 27) idg[threadIdx.x] = float(g.inv_diag[threadIdx.x]);
    const CgSeqState *s = a.st;
    if (s->done) return;  // uniform: the solve has finished
    const bool first = s->first != 0;
    const float beta = float(s->beta);
    const int parity = (int)(s->iterations & 1);
    const float *r = static_cast<const float *>(a.r);
    float *dcur = static_cast<float *>(parity ? a.d1 : a.d0);
    const float *dold = static_cast<const float *>(parity ? a.d0 : a.d1);
    float *q = static_cast<float *>(a.q);
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int t = blockIdx.x;
    const int ch = t % g.chunksp, col = t / g.chunksp;
    const int i0 = (col % g.tiles_xv) * kPipeX;
    const int j0 = (col / g.tiles_xv) * kPipeY;
    const int k0 = ch * g.kcp, k1 = min(g.nz, k0 + g.kcp);
    // staging of plane p into its ring slot (zeros outside the grid). The
    // copies a thread issues are the same for every plane, so their shared
    // offsets and in-plane global offsets (-1 outside the grid in x or y)
    // are formed once: item u copies 16 bytes of row ry (-1 .. 16) and
    // column group c4 of array arr (0 r, 1 d_old).
    auto slot_of = [&](int p) { return pipe_smem + ((p - k0 + 1) % kPipeSlots) * 2 * kPipeArr; };
    constexpr int kStageN = 2 * kPipeRows * (kPipeX / 4);
    constexpr int kStageItems = (kStageN + kBlock - 1) / kBlock;
    int soff[kStageItems], goff[kStageItems];
    unsigned dmask = 0u;  // bit u: item u copies d_old
#pragma unroll
    for (int u = 0; u < kStageItems; ++u) {
        const int e = threadIdx.x + u * kBlock;
        soff[u] = 0;
        goff[u] = -2;  // -2: no item
        if (e < kStageN) {
            const int arr = e / (kPipeRows * (kPipeX / 4)), rem = e - arr * (kPipeRows * (kPipeX / 4));
            const int ry = rem / (kPipeX / 4), c4 = rem - ry * (kPipeX / 4);
            const int j = j0 + ry - 1, i = i0 + 4 * c4;
            soff[u] = arr * kPipeArr + ry * kPipeX + 4 * c4;
            goff[u] = (j >= 0 && j < g.ny && i < g.nx) ? j * g.nx + i : -1;
            if (arr) dmask |= 1u << u;
        }
    }
    int hsoff = 0, hgoff = -2;  // the x-halo copy of threads < 4 kPipeY
    bool hd = false;
    if (threadIdx.x < 4 * kPipeY) {
        const int arr = threadIdx.x / (2 * kPipeY), side = (threadIdx.x / kPipeY) & 1, y = threadIdx.x % kPipeY;
        const int i = side ? i0 + kPipeX : i0 - 1, j = j0 + y;
        hsoff = arr * kPipeArr + kPipeRows * kPipeX + side * kPipeY + y;
        hgoff = (i >= 0 && i < g.nx && j < g.ny) ? j * g.nx + i : -1;
        hd = arr != 0;
    }
    const size_t nxy = (size_t)g.nx * g.ny;
    auto stage = [&](int p) {
        float *sl = slot_of(p);
        const bool pin = p >= 0 && p < g.nz;
        const size_t pb = pin ? (size_t)p * nxy : 0;
#pragma unroll
        for (int u = 0; u < kStageItems; ++u) {
            if (goff[u] == -2) continue;
            const bool isd = (dmask >> u) & 1u;
            const bool ok = pin && goff[u] >= 0 && !(isd && first);
            const float *base = isd ? dold : r;
            cp_async16(sl + soff[u], ok ? base + pb + goff[u] : base, ok);
        }
        if (hgoff != -2) {
            const bool ok = pin && hgoff >= 0 && !(hd && first);
            const float *base = hd ? dold : r;
            cp_async4(sl + hsoff, ok ? base + pb + hgoff : base, ok);
        }
    };
    double sdq = 0.0;
    // prologue: planes k0 - 1 .. k0 + 2 (one commit group each)
    for (int p = k0 - 1; p <= k0 + 2; ++p) {
        if (p <= k1) stage(p);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    const int ib = i0 + lane * 4;
    const bool inx = ib < g.nx;
    const int ibc = inx ? ib : 0;
    const float wx = float(g.ix2), wy = float(g.iy2), wz = float(g.iz2);
    const float wxm0 = (inx && ib > 0) ? wx : 0.f, wxpL = (inx && ib + 4 < g.nx) ? wx : 0.f;
    const int mx0 = miss(ibc, g.nx), mxL = miss(ibc + 3, g.nx);
    const bool hw = lane == 0 && i0 > 0, he = lane == 31 && i0 + kPipeX < g.nx;
    const int xh = hw ? i0 - 1 : (he ? i0 + kPipeX : 0);
    const int mxh = miss(xh, g.nx);
    const int row0 = j0 + wp * 2;  // this warp's two rows
    // The four tile rows this warp forms d on (ri 0 .. 3 = rows row0 - 1 ..
    // row0 + 2): inside the grid in y, y-class 3 miss(row), holding the
    // pinned cell (row 0, x 0).
    bool rin[4];
    int rcls[4];
    bool rpin[4];
#pragma unroll
    for (int ri = 0; ri < 4; ++ri) {
        const int row = row0 - 1 + ri;
        rin[ri] = row >= 0 && row < g.ny;
        rcls[ri] = rin[ri] ? 3 * miss(row, g.ny) : 0;
        rpin[ri] = row == 0 && ibc == 0;
    }
    // d of the lane's 4 cells of row ri of plane p from the staged raw
    // inputs; cz = miss(p, nz), pin = p inside the grid
    auto make4 = [&](const float *sl, int ri, int p, int cz, bool pin, float (&out)[4]) {
        if (!pin || !rin[ri] || !inx) {
            out[0] = out[1] = out[2] = out[3] = 0.f;
            return;
        }
        const int ry = wp * 2 - 1 + ri;
        const float4 rv = *reinterpret_cast<const float4 *>(sl + (ry + 1) * kPipeX + lane * 4);
        const float4 dv = *reinterpret_cast<const float4 *>(sl + kPipeArr + (ry + 1) * kPipeX + lane * 4);
        const float rr[4] = {rv.x, rv.y, rv.z, rv.w}, dd[4] = {dv.x, dv.y, dv.z, dv.w};
        const int cyz = rcls[ri] + cz;
        const float mid = idg[cyz];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            float id = mid;
            if (e == 0 && mx0) id = idg[9 * mx0 + cyz];
            if (e == 3 && mxL) id = idg[9 * mxL + cyz];
            const float z = rr[e] * id;
            out[e] = first ? z : float(z + beta * dd[e]);
        }
        if (p == 0 && rpin[ri]) out[0] = 0.f;  // pinned cell
    };
    auto make_halo = [&](const float *sl, int m, int p, int cz, bool pin) -> float {  // x-halo cell of own row m
        const int ri = m + 1, y = wp * 2 + m;
        if (!(hw || he) || !rin[ri] || !pin) return 0.f;
        if (p == 0 && row0 + m == 0 && xh == 0) return 0.f;
        const int side = he ? 1 : 0;
        const float rv = sl[kPipeRows * kPipeX + side * kPipeY + y];
        const float dv = sl[kPipeArr + kPipeRows * kPipeX + side * kPipeY + y];
        const float z = rv * idg[9 * mxh + rcls[ri] + cz];
        return first ? z : float(z + beta * dv);
    };
    float below[2][4], cur[2][4];
    asm volatile("cp.async.wait_group 2;" ::: "memory");  // planes k0 - 1, k0 landed
    __syncthreads();
    {
        const int pb = k0 - 1;
        const bool pinb = pb >= 0, pinc = k0 < g.nz;
        const int czb = pinb ? miss(pb, g.nz) : 0, czc = miss(k0, g.nz);
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            make4(slot_of(pb), m + 1, pb, czb, pinb, below[m]);
            make4(slot_of(k0), m + 1, k0, czc, pinc, cur[m]);
        }
    }
    for (int k = k0; k < k1; ++k) {
        if (k + 3 <= k1) stage(k + 3);
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 2;" ::: "memory");  // planes up to k + 1 landed
        __syncthreads();
        const float *slk = slot_of(k), *sla = slot_of(k + 1);
        float above[2][4], ys[4], yn[4];
        const bool pina = k + 1 < g.nz;
        const int cza = pina ? miss(k + 1, g.nz) : 0, czk = miss(k, g.nz);
        make4(sla, 1, k + 1, cza, pina, above[0]);
        make4(sla, 2, k + 1, cza, pina, above[1]);
        make4(slk, 0, k, czk, true, ys);
        make4(slk, 3, k, czk, true, yn);
        const float hx0 = make_halo(slk, 0, k, czk, true), hx1 = make_halo(slk, 1, k, czk, true);
        const float wzm = k > 0 ? wz : 0.f, wzp = k + 1 < g.nz ? wz : 0.f;
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            const int row = row0 + m;
            float west = __shfl_up_sync(0xffffffffu, cur[m][3], 1);
            float east = __shfl_down_sync(0xffffffffu, cur[m][0], 1);
            const float hxm = m ? hx1 : hx0;
            if (lane == 0) west = hw ? hxm : 0.f;
            if (lane == 31) east = he ? hxm : 0.f;
            if (!inx || row >= g.ny) continue;
            const float wym = row > 0 ? wy : 0.f, wyp = row + 1 < g.ny ? wy : 0.f;
            float dv[4], qv[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const float wxm = e == 0 ? wxm0 : wx, wxp = e == 3 ? wxpL : wx;
                const float xm = e == 0 ? west : cur[m][e > 0 ? e - 1 : 0];
                const float xp = e == 3 ? east : cur[m][e < 3 ? e + 1 : 3];
                const float ysv = m == 0 ? ys[e] : cur[0][e];
                const float ynv = m == 1 ? yn[e] : cur[1][e];
                const float c0 = cur[m][e];
                float ax = (wxm + wxp + wym + wyp + wzm + wzp) * c0 -
                           (wxm * xm + wxp * xp + wym * ysv + wyp * ynv + wzm * below[m][e] + wzp * above[m][e]);
                if (k == 0 && row == 0 && ib + e == 0) ax = c0;  // identity row of the pinned cell
                dv[e] = c0;
                qv[e] = ax;
                sdq += double(c0) * double(ax);
            }
            const size_t c = ((size_t)k * g.ny + row) * g.nx + ib;
            *reinterpret_cast<float4 *>(dcur + c) = make_float4(dv[0], dv[1], dv[2], dv[3]);
            *reinterpret_cast<float4 *>(q + c) = make_float4(qv[0], qv[1], qv[2], qv[3]);
        }
#pragma unroll
        for (int m = 0; m < 2; ++m)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                below[m][e] = cur[m][e];
                cur[m][e] = above[m][e];
            }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    const double v[1] = {sdq};
    if (!reduce_arrive<1>(v, a.partials, &a.st->counter, red)) return;
    double o[1];
    reduce_finish<1>(o, a.partials, red);
    if (threadIdx.x == 0) {
        CgSeqState *w = a.st;
        w->counter = 0;
        const double dq = o[0];
        if (fabs(dq) < 1.0e-30 || !isfinite(dq) || !isfinite(w->rz_old / dq)) {
            w->error = FLURSYS_ERR_BREAKDOWN;
            w->done = 1;
            w->alpha = 0.0;
        } else {
            w->alpha = w->rz_old / dq;
        }
    }
}

template <typename V, bool MIXED>
__global__ void __launch_bounds__(kBlock) seq_update(SeqArgs a) {
    __shared__ double red[kSlots * (kBlock / 32)];
    const CgSeqState *s = a.st;
    if (s->done) {
        // The solve has finished: host-driven mode, a later iteration of an
        // unrolled body, or a breakdown found by this iteration's operand
        // kernel (which sets `done` and leaves the conditions to this kernel).
        // Either way no replacement and no further iteration.
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            set_cond(a, a.h_replace, 0u);
            set_cond(a, a.h_loop, 0u);
        }
        return;
    }
    const double alpha = s->alpha;
    const bool dead = s->error != 0;
    const int parity = (int)(s->iterations & 1);
    V *r = static_cast<V *>(a.r);
    const V *dcur = static_cast<const V *>(parity ? a.d1 : a.d0);
    const V *q = static_cast<const V *>(a.q);
    const SeqGeo &g = a.g;
    double srr = 0.0, srz = 0.0, smax = 0.0;
    if (!dead) {
        using V4 = typename std::conditional<std::is_same<V, float>::value, float4, double2>::type;
        constexpr int W = sizeof(V4) / sizeof(V);
        const int nrow = g.nx / W;
        const bool vec = (g.nx % W) == 0;
        const int nv = vec ? g.ny * g.nz * nrow : 0;
        const int stride = gridDim.x * kBlock;
        for (int cv = blockIdx.x * kBlock + threadIdx.x; cv < nv; cv += stride) {
            const int row = cv / nrow;
            const int i0 = (cv - row * nrow) * W;
            const int c0 = cv * W;
            const int rcls = a.row_class[row];
            const V4 d4 = reinterpret_cast<const V4 *>(dcur)[cv];
            const V4 q4 = reinterpret_cast<const V4 *>(q)[cv];
            V4 r4 = reinterpret_cast<const V4 *>(r)[cv];
            const V *dv = reinterpret_cast<const V *>(&d4);
            const V *qv = reinterpret_cast<const V *>(&q4);
            V *rv = reinterpret_cast<V *>(&r4);
            if (MIXED) {
                float4 x4 = reinterpret_cast<const float4 *>(a.dx)[cv];
                float *xv = reinterpret_cast<float *>(&x4);
#pragma unroll
                for (int e = 0; e < W; ++e) xv[e] = float(double(xv[e]) + alpha * double(dv[e]));
                reinterpret_cast<float4 *>(a.dx)[cv] = x4;
            } else {
                double2 *xp = reinterpret_cast<double2 *>(a.x + c0);
                double2 x2 = *xp;
                x2.x += (c0 == 0) ? 0.0 : alpha * double(dv[0]);
                x2.y += alpha * double(dv[1]);
                *xp = x2;
            }
            const double idg_mid = g.inv_diag[rcls];
#pragma unroll
            for (int e = 0; e < W; ++e) {
                rv[e] = V(double(rv[e]) - alpha * double(qv[e]));
                const double rd = double(rv[e]);
                const int ie = i0 + e;
                const double idg = (ie == 0 || ie == g.nx - 1) ? g.inv_diag[9 * miss(ie, g.nx) + rcls] : idg_mid;
                srr += rd * rd;
                srz += rd * rd * ((c0 + e == 0) ? 1.0 : idg);
                smax = fmax(smax, fabs(rd));
            }
            reinterpret_cast<V4 *>(r)[cv] = r4;
        }
        const int ns = vec ? 0 : g.n;
        for (int c = blockIdx.x * kBlock + threadIdx.x; c < ns; c += stride) {
            const int row = c / g.nx;
            const int i = c - row * g.nx;
            const double dcv = double(dcur[c]);
            if (MIXED) a.dx[c] = float(double(a.dx[c]) + alpha * dcv);
            else if (c != 0) a.x[c] += alpha * dcv;
            const V rv = V(double(r[c]) - alpha * double(q[c]));
            r[c] = rv;
            const double rd = double(rv);
            srr += rd * rd;
            srz += rd * rd * (c == 0 ? 1.0 : g.inv_diag[9 * miss(i, g.nx) + a.row_class[row]]);
            smax = fmax(smax, fabs(rd));
        }
    }
    const double v[3] = {srr, srz, smax};
    if (!reduce_arrive<3>(v, a.partials, &a.st->counter, red)) return;
    double o[3];
    reduce_finish<3>(o, a.partials, red);
    if (threadIdx.x == 0) {
        CgSeqState *w = a.st;
        w->counter = 0;
        if (w->error) {
            w->done = 1;
            set_cond(a, a.h_replace, 0u);
            set_cond(a, a.h_loop, 0u);
            return;
        }
        w->iterations += 1;
        const bool l2 = a.stop_rule == FLURSYS_STOP_REL_L2;
        const double res = l2 ? sqrt(o[0]) : o[2];
        w->residual = res;
        if (!isfinite(res)) {
            w->error = FLURSYS_ERR_NON_FINITE;
            w->done = 1;
            set_cond(a, a.h_replace, 0u);
            set_cond(a, a.h_loop, 0u);
            return;
        }
        const bool conv = stop_ok(a, res, w->threshold);
        const bool replace = MIXED && (conv || (w->iterations % a.replace_every) == 0);
        if (replace) {
            w->replace = 1;
            w->rz_new = o[1];
            set_cond(a, a.h_replace, 1u);
            return;  // the replacement launch takes the decision
        }
        set_cond(a, a.h_replace, 0u);
        if (conv) {
            w->status = FLURSYS_LINEAR_CONVERGED;
            w->done = 1;
        } else if (fabs(w->rz_old) < 1.0e-30 || w->iterations >= a.max_iters) {
            w->done = 1;
        } else {
            w->beta = o[1] / w->rz_old;
            w->rz_old = o[1];
            w->first = 0;
        }
        set_cond(a, a.h_loop, w->done ? 0u : 1u);
    }
}

__global__ void __launch_bounds__(kBlock) seq_fold(SeqArgs a) {
    if (!a.graph && !a.st->replace) return;  // host-driven mode: no replacement due
    const int stride = gridDim.x * kBlock;
    for (int c = blockIdx.x * kBlock + threadIdx.x; c < a.g.n; c += stride) {
        if (c == 0) { a.x[0] = 0.0; continue; }
        a.x[c] += double(a.dx[c]);
    }
}

template <typename V, bool MIXED>
__global__ void __launch_bounds__(kBlock) seq_replace(SeqArgs a) {
    __shared__ double tile[(TY + 2) * (TX + 2)];
    __shared__ double red[kSlots * (kBlock / 32)];
    if (!a.graph && !a.st->replace) return;  // host-driven mode: no replacement due
    double srr = 0.0, srz = 0.0, smax = 0.0;
    residual_tile<V, MIXED>(a, static_cast<V *>(a.r), tile, srr, srz, smax, true);
    const double v[3] = {srr, srz, smax};
    if (!reduce_arrive<3>(v, a.partials, &a.st->counter, red)) return;
    double o[3];
    reduce_finish<3>(o, a.partials, red);
    if (threadIdx.x == 0) {
        CgSeqState *w = a.st;
        w->counter = 0;
        w->replace = 0;
        const bool l2 = a.stop_rule == FLURSYS_STOP_REL_L2;
        const double res = l2 ? sqrt(o[0]) : o[2];
        w->residual = res;
        if (!isfinite(res)) {
            w->error = FLURSYS_ERR_NON_FINITE;
            w->done = 1;
        } else if (stop_ok(a, res, w->threshold)) {
            w->status = FLURSYS_LINEAR_CONVERGED;
            w->done = 1;
        } else if (fabs(w->rz_old) < 1.0e-30 || w->iterations >= a.max_iters) {
            w->done = 1;
        } else {
            w->beta = o[1] / w->rz_old;
            w->rz_old = o[1];
            w->first = 0;
        }
        set_cond(a, a.h_loop, w->done ? 0u : 1u);
    }
}

// Folds a pending increment (MIXED, not converged), then ||b - A x||_2.
template <typename V, bool MIXED>
__global__ void __launch_bounds__(kBlock) seq_final(SeqArgs a) {
    __shared__ double tile[(TY + 2) * (TX + 2)];
    __shared__ double red[kSlots * (kBlock / 32)];
    double s_true = 0.0;
    tile_sweep(
        a.g, blockIdx.x, tile, [&](int c) -> double { return a.x[c]; },
        [&](double v, int, bool pin) -> double { return pin ? 0.0 : v; },
        [&](int c, int, bool pin, double, double ax) {
            const double t = pin ? 0.0 : -__ldg(a.rhs + c) - ax;
            s_true += t * t;
        });
    const double v[1] = {s_true};
    if (!reduce_arrive<1>(v, a.partials, &a.st->counter, red)) return;
    double o[1];
    reduce_finish<1>(o, a.partials, red);
    if (threadIdx.x == 0) {
        a.st->counter = 0;
        a.st->true_l2 = sqrt(o[0]);
    }
}

// MIXED: fold the increment left over when the loop stops without a final
// replacement (iteration limit or breakdown).
__global__ void __launch_bounds__(kBlock) seq_fold_pending(SeqArgs a) {
    const CgSeqState *s = a.st;
    if (s->status == FLURSYS_LINEAR_CONVERGED) return;
    const int stride = gridDim.x * kBlock;
    for (int c = blockIdx.x * kBlock + threadIdx.x; c < a.g.n; c += stride) {
        if (c == 0) { a.x[0] = 0.0; continue; }
        a.x[c] += double(a.dx[c]);
        a.dx[c] = 0.f;
    }
}

// ---------------------------------------------------------------------------
// Single-reduction PCG (MIXED): one stencil launch per iteration.
//
// The vectors are those of the standard PCG (u = M r with M the Jacobi
// inverse, p_i = u_i + beta_{i-1} p_{i-1}, s_i = A p_i, x += alpha_i p_i,
// r_{i+1} = r_i - alpha_i s_i), computed in the same precisions; only the
// scalars are rearranged so that an iteration needs one global reduction.
// The launch of iteration i also forms u_{i+1} and w_{i+1} = A u_{i+1}, and
// the denominator of the next step is expanded exactly (A symmetric on the
// unpinned cells, where p and u live):
//   (p_{i+1}, A p_{i+1}) = delta + 2 b e + b^2 f,
//   delta = (u_{i+1}, w_{i+1}), e = (u_{i+1}, s_i), f = (p_i, s_i),
// with b = beta_i rounded to FP32 as in the formation of p_{i+1}. So one
// sweep yields gamma_{i+1} = r.M r, ||r||, max|r|, delta, e, f; its last
// block sets beta_i = gamma_{i+1} / gamma_i and alpha_{i+1}.
//
// w needs u_{i+1} one cell around a cell, u_{i+1} needs s_i there, and s_i
// needs p_i one cell further. Each block owns a 32 x 8 x TZ tile: one TMA box
// load brings r_i and p_{i-1} on the tile plus two cells (R2; the box starts
// four cells early in x for 16-byte alignment, and the hardware fills cells
// outside the grid with zeros) and dx of the tile into shared memory; then,
// separated by block barriers, p_i on R2 (in place), s_i, r_{i+1} and u_{i+1}
// on the tile plus one cell (R1; u replaces r in place, the owned cells write
// r, p and dx to the other buffer set), and w = A u on the tile. Halo values
// repeat the owners' arithmetic with the same correctly rounded operations
// (explicit fma / mul intrinsics), so they are bit-identical. r and p
// alternate between two buffer sets (set iterations & 1 is read, the other
// written). Per iteration a cell costs 24 B of compulsory traffic (read r, p,
// dx; write r, p, dx) against 40 B for the two-launch form; the halo re-reads
// are served by L2. Needs nx % 4 == 0 (TMA row stride); other grids take the
// two-launch form.
// The FP64 residual replacement (every `replace_every` iterations and before
// accepting convergence) folds dx into x, recomputes r = b - A x, then delta,
// e and f of the replaced state.
// ---------------------------------------------------------------------------
// 7-point operator row with a fixed operation order.
__device__ __forceinline__ float cg1_row(float c, float xm, float xp, float ym, float yp, float zm, float zp, float wxm,
                                         float wxp, float wym, float wyp, float wzm, float wzp) {
    const float dg = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(wxm, wxp), wym), wyp), wzm), wzp);
    float nb = __fmul_rn(wxm, xm);
    nb = __fmaf_rn(wxp, xp, nb);
    nb = __fmaf_rn(wym, ym, nb);
    nb = __fmaf_rn(wyp, yp, nb);
    nb = __fmaf_rn(wzm, zm, nb);
    nb = __fmaf_rn(wzp, zp, nb);
    return __fmaf_rn(dg, c, -nb);
}

// beta_i and alpha_{i+1} from the sums of an iteration (or of a replacement);
// marks the solve done on the iteration cap or a breakdown.
__device__ __forceinline__ void cg1_next(const SeqArgs &a, CgSeqState *w, double gam, double del, double e,
                                         double f) {
    if (fabs(w->rz_old) < 1.0e-30 || w->iterations >= a.max_iters) {
        w->done = 1;
        return;
    }
    const double beta = gam / w->rz_old;
    const double bf = double(float(beta));  // p_{i+1} = u + float(beta) p_i
    const double den = del + 2.0 * bf * e + bf * bf * f;
    const double alpha = gam / den;
    if (fabs(den) < 1.0e-30 || !isfinite(den) || !isfinite(alpha)) {
        w->error = FLURSYS_ERR_BREAKDOWN;
        w->done = 1;
        w->alpha = 0.0;
        return;
    }
    w->beta = beta;
    w->alpha = alpha;
    w->rz_old = gam;
    w->first = 0;
}

// Last block of a step launch: o = {gamma, ||r||^2, e, f, delta}, mx = max|r|.
__device__ __forceinline__ void cg1_step_finish(const SeqArgs &a, const double (&o)[5], double mx) {
    CgSeqState *w = a.st;
    w->counter = 0;
    w->iterations += 1;
    const bool l2 = a.stop_rule == FLURSYS_STOP_REL_L2;
    const double res = l2 ? sqrt(o[1]) : mx;
    w->residual = res;
    if (!isfinite(res)) {
        w->error = FLURSYS_ERR_NON_FINITE;
        w->done = 1;
        set_cond(a, a.h_replace, 0u);
        set_cond(a, a.h_loop, 0u);
        return;
    }
    const bool conv = stop_ok(a, res, w->threshold);
    if (conv || (w->iterations % a.replace_every) == 0) {
        w->replace = 1;
        w->rz_new = o[0];
        set_cond(a, a.h_replace, 1u);
        return;  // the replacement launches take the decision
    }
    set_cond(a, a.h_replace, 0u);
    cg1_next(a, w, o[0], o[4], o[2], o[3]);
    set_cond(a, a.h_loop, w->done ? 0u : 1u);
}

// Tensor maps of the step kernel: r and p (both buffer sets) with the halo
// box, dx with the tile box.
struct Cg1Maps {
    CUtensorMap r[2], p[2], dx;
};

template <int TZ>
struct Cg1Tile {
    static constexpr int BX = TX + 8, BY = TY + 4, BZ = TZ + 4;  // halo box (x from i0 - 4)
    static constexpr int PL = BX * BY;                            // one box plane
    static constexpr int BOX = PL * BZ;
    static constexpr int TILE = TX * TY * TZ;
    static constexpr size_t smem_bytes = sizeof(float) * (2 * BOX + TILE) + 128;  // + alignment slack
};

constexpr long long kTmaWaitLimit = 4'000'000LL;  // polls of ~64 ns: well above any legitimate wait

// The step kernel (one launch per iteration).
template <int TZ>
__global__ void __launch_bounds__(kBlock, 4) cg1_tile(const __grid_constant__ SeqArgs a, const __grid_constant__ Cg1Maps m) {
    using L = Cg1Tile<TZ>;
    constexpr int BX = L::BX, PL = L::PL;
    extern __shared__ unsigned char dyn[];
    float *Rs = reinterpret_cast<float *>((reinterpret_cast<uintptr_t>(dyn) + 127) & ~uintptr_t(127));
    float *Ps = Rs + L::BOX;
    float *Ds = Ps + L::BOX;
    __shared__ __align__(8) uint64_t bar;
    __shared__ float idg[27];
    __shared__ double red[kSlots * (kBlock / 32)];
    __shared__ int s_bad;
    const SeqGeo &g = a.g;
    const CgSeqState *st = a.st;
    if (!a.graph && st->done) return;  // host-driven mode: the solve has finished
    const double alpha = st->alpha;
    const float vbeta = float(st->beta);
    const bool first = st->first != 0;
    const int par = (int)(st->iterations & 1);
    float *rB = par ? a.cr[0] : a.cr[1];
    float *pB = par ? a.cp[0] : a.cp[1];
    float *dxv = a.dx;
    const int bid = blockIdx.x;
    const int i0 = (bid % g.tiles_x) * TX;
    const int j0 = ((bid / g.tiles_x) % g.tiles_y) * TY;
    const int k0 = (bid / (g.tiles_x * g.tiles_y)) * TZ;
    const int tid = threadIdx.x;
    if (tid < 27) idg[tid] = float(g.inv_diag[tid]);
    if (tid == 0) {
        s_bad = 0;
        mbar_init(&bar, 1);
    }
    __syncthreads();
    if (tid == 0) {
        mbar_expect_tx(&bar, sizeof(float) * ((first ? 1 : 2) * L::BOX + L::TILE));
        tma_load_3d(Rs, &m.r[par], i0 - 4, j0 - 2, k0 - 2, &bar);
        if (!first) tma_load_3d(Ps, &m.p[par], i0 - 4, j0 - 2, k0 - 2, &bar);
        tma_load_3d(Ds, &m.dx, i0, j0, k0, &bar);
    }
    if (!mbar_wait_bounded(&bar, 0, kTmaWaitLimit)) {
        s_bad = 1;
        mbar_wait_bounded(&bar, 0, kTmaWaitLimit);  // let copies in flight land before the block moves on
    }
    __syncthreads();
    const bool bad = s_bad != 0;
    const float wx = float(g.ix2), wy = float(g.iy2), wz = float(g.iz2);
    double sg = 0.0, srr = 0.0, smx = 0.0, se = 0.0, sf = 0.0, sd = 0.0;
    if (!bad) {
        // z class of each box plane (missing neighbours in z), shared by all columns
        auto zmiss = [&](int gk) { return miss(gk, g.nz); };
        // (1) p_i on R2: columns -2..33, rows -2..9, planes -2..TZ+1 of the
        // tile. The pinned cell needs no case: r = 0 and p_{i-1} = 0 there.
        for (int q = tid; q < (TX + 4) * (TY + 4); q += kBlock) {
            const int x = q % (TX + 4), y = q / (TX + 4);
            const int gi = i0 - 2 + x, gj = j0 - 2 + y;
            const float *idc = idg + 9 * miss(gi, g.nx) + 3 * miss(gj, g.ny);
            const int s0 = y * BX + x + 2;
#pragma unroll
            for (int z = 0; z < TZ + 4; ++z) {
                const int sc = z * PL + s0;
                const float u = __fmul_rn(Rs[sc], idc[zmiss(k0 - 2 + z)]);
                Ps[sc] = first ? u : __fmaf_rn(vbeta, Ps[sc], u);
            }
        }
        __syncthreads();
        // (2) s_i = A p_i, r_{i+1}, u_{i+1} on R1: columns -1..32, rows -1..8,
        // planes -1..TZ; owned cells write r_{i+1}, p_i, dx and their sums.
        // The pinned cell's identity row gives s = p = 0 there, hence r and u
        // stay 0.
        for (int q = tid; q < (TX + 2) * (TY + 2); q += kBlock) {
            const int x = q % (TX + 2), y = q / (TX + 2);
            const int gi = i0 - 1 + x, gj = j0 - 1 + y;
            const bool inxy = gi >= 0 && gi < g.nx && gj >= 0 && gj < g.ny;
            const float wxm = inxy && gi > 0 ? wx : 0.f, wxp = inxy && gi + 1 < g.nx ? wx : 0.f;
            const float wym = inxy && gj > 0 ? wy : 0.f, wyp = inxy && gj + 1 < g.ny ? wy : 0.f;
            const float *idc = idg + 9 * miss(gi, g.nx) + 3 * miss(gj, g.ny);
            const bool pcol = gi == 0 && gj == 0;
            const bool own_xy = inxy && x >= 1 && x <= TX && y >= 1 && y <= TY;
            const int s0 = (y + 1) * BX + x + 3;
            const int cg0 = own_xy ? gj * g.nx + gi : 0;
            const float *dsc = Ds + (y - 1) * TX + (x - 1);
            float pb = Ps[s0], pc = Ps[PL + s0];
#pragma unroll
            for (int z = 0; z < TZ + 2; ++z) {
                const int gk = k0 - 1 + z;
                const int sc = (z + 1) * PL + s0;
                const float pa = Ps[sc + PL];
                const bool inz = gk >= 0 && gk < g.nz;
                const float wzm = inz && gk > 0 ? wz : 0.f, wzp = inz && gk + 1 < g.nz ? wz : 0.f;
                float s = cg1_row(pc, Ps[sc - 1], Ps[sc + 1], Ps[sc - BX], Ps[sc + BX], pb, pa, wxm, wxp, wym, wyp, wzm,
                                  wzp);
                if (pcol && gk == 0) s = 0.f;
                const float rn = float(__fma_rn(-alpha, double(s), double(Rs[sc])));
                const float id = idc[zmiss(gk)];
                const float u = __fmul_rn(rn, id);
                if (z >= 1 && z <= TZ && own_xy && inz) {
                    const int c = cg0 + gk * g.nxy;
                    rB[c] = rn;
                    pB[c] = pc;
                    dxv[c] = float(double(dsc[(z - 1) * TX * TY]) + alpha * double(pc));
                    const double rd = rn;
                    sg += rd * rd * double(id);
                    srr += rd * rd;
                    smx = fmax(smx, fabs(rd));
                    se += double(u) * double(s);
                    sf += double(pc) * double(s);
                }
                Rs[sc] = u;  // read at this cell only in this phase
                pb = pc;
                pc = pa;
            }
        }
        __syncthreads();
        // (3) w = A u_{i+1} on the tile: delta (the pinned row is the identity, w = u = 0)
        {
            const int x = tid % TX, y = tid / TX;
            const int gi = i0 + x, gj = j0 + y;
            if (gi < g.nx && gj < g.ny) {
                const float wxm = gi > 0 ? wx : 0.f, wxp = gi + 1 < g.nx ? wx : 0.f;
                const float wym = gj > 0 ? wy : 0.f, wyp = gj + 1 < g.ny ? wy : 0.f;
                const bool pcol = gi == 0 && gj == 0;
                const int s0 = (y + 2) * BX + x + 4;
                float ub = Rs[PL + s0], uc = Rs[2 * PL + s0];
#pragma unroll
                for (int z = 0; z < TZ; ++z) {
                    const int gk = k0 + z;
                    const int sc = (z + 2) * PL + s0;
                    const float ua = Rs[sc + PL];
                    const float wzm = gk > 0 ? wz : 0.f, wzp = gk + 1 < g.nz ? wz : 0.f;
                    float w = cg1_row(uc, Rs[sc - 1], Rs[sc + 1], Rs[sc - BX], Rs[sc + BX], ub, ua, wxm, wxp, wym, wyp,
                                      wzm, wzp);
                    if (pcol && gk == 0) w = 0.f;
                    if (gk < g.nz) sd += double(uc) * double(w);
                    ub = uc;
                    uc = ua;
                }
            }
        }
    }
    if (bad && tid == 0) atomicExch(&a.st->error, (int)FLURSYS_ERR_TIMEOUT);
    double v[5] = {sg, srr, se, sf, sd};
    if (!arrive_n<5, true>(v, smx, a.partials, &a.st->counter, red)) return;
    double o[5], mx;
    finish_n<5, true>(o, mx, a.partials, red);
    if (threadIdx.x == 0) {
        CgSeqState *w = a.st;
        if (w->error) {
            w->counter = 0;
            w->done = 1;
            set_cond(a, a.h_replace, 0u);
            set_cond(a, a.h_loop, 0u);
            return;
        }
        cg1_step_finish(a, o, mx);
    }
}

// FP64 residual replacement of the single-reduction variant: r = b - A x into
// the set the next step reads (x already holds the folded increment).
__global__ void __launch_bounds__(kBlock) cg1_replace_r(SeqArgs a) {
    __shared__ double tile[(TY + 2) * (TX + 2)];
    __shared__ double red[kSlots * (kBlock / 32)];
    if (!a.graph && a.st->replace != 1) return;  // host-driven mode: no replacement due
    float *r = (a.st->iterations & 1) ? a.cr[1] : a.cr[0];
    double srr = 0.0, srz = 0.0, smax = 0.0;
    residual_tile<float, true>(a, r, tile, srr, srz, smax, true);
    const double v[3] = {srr, srz, smax};
    if (!reduce_arrive<3>(v, a.partials, &a.st->counter, red)) return;
    double o[3];
    reduce_finish<3>(o, a.partials, red);
    if (threadIdx.x == 0) {
        CgSeqState *w = a.st;
        w->counter = 0;
        const bool l2 = a.stop_rule == FLURSYS_STOP_REL_L2;
        const double res = l2 ? sqrt(o[0]) : o[2];
        w->residual = res;
        if (!isfinite(res)) {
            w->error = FLURSYS_ERR_NON_FINITE;
            w->done = 1;
        } else if (stop_ok(a, res, w->threshold)) {
            w->status = FLURSYS_LINEAR_CONVERGED;
            w->done = 1;
        } else if (fabs(w->rz_old) < 1.0e-30 || w->iterations >= a.max_iters) {
            w->done = 1;
        } else {
            w->rz_new = o[1];
        }
        w->replace = w->done ? 0 : 2;
        set_cond(a, a.h_loop, w->done ? 0u : 1u);
    }
}

// delta = (u, A u) with u = M r of the current set, and with MODE 1 also
// e = (u, A p) and f = (p, A p) of the current p; then the step
// coefficients. MODE 0 follows the initial residual (alpha_0 = gamma_0 /
// delta_0, p_0 = u_0), MODE 1 a residual replacement.
template <int MODE>
__global__ void __launch_bounds__(kBlock) cg1_ws(SeqArgs a) {
    __shared__ double tile[(TY + 2) * (TX + 2)];
    __shared__ double red[kSlots * (kBlock / 32)];
    const CgSeqState *st = a.st;
    if (st->done) return;                                   // converged at the start or the replacement
    if (MODE == 1 && !a.graph && st->replace != 2) return;  // host-driven mode: no replacement due
    const bool par = (st->iterations & 1) != 0;
    const float *r = par ? a.cr[1] : a.cr[0];
    const float *p = par ? a.cp[1] : a.cp[0];
    const SeqGeo &g = a.g;
    double sd = 0.0, se = 0.0, sf = 0.0;
    tile_sweep(
        g, blockIdx.x, tile, [&](int c) -> float { return r[c]; },
        [&](float v, int cls, bool pin) -> float { return pin ? 0.f : __fmul_rn(v, float(g.inv_diag[cls])); },
        [&](int, int, bool, float u, float w) { sd += double(u) * double(w); });
    if (MODE == 1) {
        tile_sweep(
            g, blockIdx.x, tile, [&](int c) -> float { return p[c]; },
            [&](float v, int, bool pin) -> float { return pin ? 0.f : v; },
            [&](int c, int cls, bool pin, float pc, float s) {
                const float u = pin ? 0.f : __fmul_rn(r[c], float(g.inv_diag[cls]));
                se += double(u) * double(s);
                sf += double(pc) * double(s);
            });
    }
    double v[3] = {sd, se, sf};
    if (!arrive_n<3, false>(v, 0.0, a.partials, &a.st->counter, red)) return;
    double o[3], mx;
    finish_n<3, false>(o, mx, a.partials, red);
    if (threadIdx.x == 0) {
        CgSeqState *w = a.st;
        w->counter = 0;
        if (MODE == 0) {
            const double alpha = w->rz_old / o[0];
            if (fabs(o[0]) < 1.0e-30 || !isfinite(o[0]) || !isfinite(alpha)) {
                w->error = FLURSYS_ERR_BREAKDOWN;
                w->done = 1;
                w->alpha = 0.0;
                set_cond(a, a.h_loop, 0u);
            } else {
                w->alpha = alpha;
            }
        } else {
            w->replace = 0;
            cg1_next(a, w, w->rz_new, o[0], o[1], o[2]);
            set_cond(a, a.h_loop, w->done ? 0u : 1u);
        }
    }
}

cudaError_t add_kernel(cudaGraph_t g, cudaGraphNode_t *node, const cudaGraphNode_t *deps, size_t ndeps,
                       const void *fn, int grid, void **args, unsigned smem = 0) {
    cudaKernelNodeParams p{};
    p.func = const_cast<void *>(fn);
    p.gridDim = dim3(grid);
    p.blockDim = dim3(kBlock);
    p.sharedMemBytes = smem;
    p.kernelParams = args;
    p.extra = nullptr;
    return cudaGraphAddKernelNode(node, g, deps, ndeps, &p);
}

template <typename V, bool MIXED>
cudaError_t build(Pcg3dSeqPlan &plan, SeqArgs &a) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaGraphCreate(&g, 0);
    if (e != cudaSuccess) return e;
    plan.graph = g;
    cudaGraphConditionalHandle hl;
    e = cudaGraphConditionalHandleCreate(&hl, g, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return e;
    a.h_loop = hl;
    // WHILE node first, so that the IF handle of its body exists before any
    // kernel node copies the argument block.
    cudaGraphNodeParams wp{};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = hl;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t n_while;
    e = cudaGraphAddNode(&n_while, g, nullptr, 0, &wp);
    if (e != cudaSuccess) return e;
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    // The body holds `unroll` iterations (FLURSYS_PCG_UNROLL, default 8;
    // measured on B200 at 128^3: 39.7 / 38.2 / 37.4 ms per step for 1 / 2 /
    // 4 on one box, 37.07 / 36.75 ms for 4 / 8 on another), so the loop
    // condition is evaluated once per `unroll` iterations;
    // the kernels of an iteration that follows the end of the solve return at
    // once (and clear the conditions). Each IF node has its own handle, set
    // by the pointwise kernel before it.
    int unroll = 8;
    if (const char *env = std::getenv("FLURSYS_PCG_UNROLL")) unroll = std::max(1, std::min(8, std::atoi(env)));
    cudaGraphNode_t n_init, n_final;
    void *args[] = {&a};
    e = add_kernel(g, &n_init, nullptr, 0, (const void *)seq_init<V, MIXED>, a.nblocks_stencil, args);
    if (e == cudaSuccess) e = cudaGraphAddDependencies(g, &n_init, &n_while, 1);
    if (e != cudaSuccess) return e;
    const void *dir_fn = a.sweep == kSweepVec    ? (const void *)seq_dir_vec<V, MIXED, kRyVec>
                         : (MIXED && a.sweep == kSweepPipe) ? (const void *)seq_dir_pipe
                                                            : (const void *)seq_dir_spmv<V, MIXED>;
    const unsigned dir_smem = (MIXED && a.sweep == kSweepPipe) ? (unsigned)kPipeSmem : 0u;
    cudaGraphNode_t prev{};
    for (int u = 0; u < unroll; ++u) {
        cudaGraphConditionalHandle hr;
        e = cudaGraphConditionalHandleCreate(&hr, body, 0, cudaGraphCondAssignDefault);
        if (e != cudaSuccess) return e;
        SeqArgs au = a;
        au.h_replace = hr;
        if (u == 0) a.h_replace = hr;  // the argument block of the nodes outside the body
        void *uargs[] = {&au};
        cudaGraphNode_t n_dir, n_upd, n_if;
        e = add_kernel(body, &n_dir, u ? &prev : nullptr, u ? 1 : 0, dir_fn, a.nblocks_dir, uargs, dir_smem);
        if (e == cudaSuccess)
            e = add_kernel(body, &n_upd, &n_dir, 1, (const void *)seq_update<V, MIXED>, a.nblocks_point, uargs);
        if (e != cudaSuccess) return e;
        cudaGraphNodeParams ip{};
        ip.type = cudaGraphNodeTypeConditional;
        ip.conditional.handle = hr;
        ip.conditional.type = cudaGraphCondTypeIf;
        ip.conditional.size = 1;
        e = cudaGraphAddNode(&n_if, body, &n_upd, 1, &ip);
        if (e != cudaSuccess) return e;
        cudaGraph_t rb = ip.conditional.phGraph_out[0];
        if (MIXED) {
            cudaGraphNode_t n_fold, n_rep;
            e = add_kernel(rb, &n_fold, nullptr, 0, (const void *)seq_fold, a.nblocks_point, uargs);
            if (e == cudaSuccess)
                e = add_kernel(rb, &n_rep, &n_fold, 1, (const void *)seq_replace<V, MIXED>, a.nblocks_stencil, uargs);
        } else {
            cudaGraphNode_t n_empty;
            e = cudaGraphAddEmptyNode(&n_empty, rb, nullptr, 0);
        }
        if (e != cudaSuccess) return e;
        prev = n_if;
    }
    cudaGraphNode_t after = n_while;
    if (MIXED) {
        cudaGraphNode_t n_pend;
        e = add_kernel(g, &n_pend, &n_while, 1, (const void *)seq_fold_pending, a.nblocks_point, args);
        if (e != cudaSuccess) return e;
        after = n_pend;
    }
    e = add_kernel(g, &n_final, &after, 1, (const void *)seq_final<V, MIXED>, a.nblocks_stencil, args);
    if (e != cudaSuccess) return e;
    return cudaGraphInstantiate(&plan.exec, g, 0);
}

// Graph of the single-reduction variant (MIXED):
//   init -> ws<0> -> WHILE(continue) { step -> IF(replace) { fold -> replace_r -> ws<1> } }
//        -> fold_pending -> final
cudaError_t build_cg1(Pcg3dSeqPlan &plan, SeqArgs &a, const Cg1Maps &maps) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaGraphCreate(&g, 0);
    if (e != cudaSuccess) return e;
    plan.graph = g;
    cudaGraphConditionalHandle hl;
    e = cudaGraphConditionalHandleCreate(&hl, g, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return e;
    a.h_loop = hl;
    cudaGraphNodeParams wp{};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = hl;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t n_while;
    e = cudaGraphAddNode(&n_while, g, nullptr, 0, &wp);
    if (e != cudaSuccess) return e;
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    cudaGraphConditionalHandle hr;
    e = cudaGraphConditionalHandleCreate(&hr, body, 0, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return e;
    a.h_replace = hr;
    void *args[] = {&a};
    cudaGraphNode_t n_init, n_prime, n_step, n_if, n_pend, n_final;
    e = add_kernel(g, &n_init, nullptr, 0, (const void *)seq_init<float, true>, a.nblocks_stencil, args);
    if (e == cudaSuccess) e = add_kernel(g, &n_prime, &n_init, 1, (const void *)cg1_ws<0>, a.nblocks_stencil, args);
    if (e == cudaSuccess) e = cudaGraphAddDependencies(g, &n_prime, &n_while, 1);
    {
        void *step_args[] = {&a, const_cast<Cg1Maps *>(&maps)};
        const void *fn = a.cg1_tz == 4 ? (const void *)cg1_tile<4> : (const void *)cg1_tile<8>;
        const unsigned smem = (unsigned)(a.cg1_tz == 4 ? Cg1Tile<4>::smem_bytes : Cg1Tile<8>::smem_bytes);
        if (e == cudaSuccess) e = add_kernel(body, &n_step, nullptr, 0, fn, a.nblocks_cg1, step_args, smem);
    }
    if (e != cudaSuccess) return e;
    cudaGraphNodeParams ip{};
    ip.type = cudaGraphNodeTypeConditional;
    ip.conditional.handle = hr;
    ip.conditional.type = cudaGraphCondTypeIf;
    ip.conditional.size = 1;
    e = cudaGraphAddNode(&n_if, body, &n_step, 1, &ip);
    if (e != cudaSuccess) return e;
    cudaGraph_t rb = ip.conditional.phGraph_out[0];
    cudaGraphNode_t n_fold, n_rep, n_ws;
    e = add_kernel(rb, &n_fold, nullptr, 0, (const void *)seq_fold, a.nblocks_point, args);
    if (e == cudaSuccess) e = add_kernel(rb, &n_rep, &n_fold, 1, (const void *)cg1_replace_r, a.nblocks_stencil, args);
    if (e == cudaSuccess) e = add_kernel(rb, &n_ws, &n_rep, 1, (const void *)cg1_ws<1>, a.nblocks_stencil, args);
    if (e == cudaSuccess) e = add_kernel(g, &n_pend, &n_while, 1, (const void *)seq_fold_pending, a.nblocks_point, args);
    if (e == cudaSuccess)
        e = add_kernel(g, &n_final, &n_pend, 1, (const void *)seq_final<float, true>, a.nblocks_stencil, args);
    if (e != cudaSuccess) return e;
    return cudaGraphInstantiate(&plan.exec, g, 0);
}

}  // namespace

cudaError_t pcg3d_seq_plan(Pcg3dSeqPlan &plan, const Pcg3dArgs &args, int precision, int device) {
    pcg3d_seq_destroy(plan);
    SeqArgs a{};
    SeqGeo &g = a.g;
    g.nx = args.nx; g.ny = args.ny; g.nz = args.nz;
    g.nxy = args.nx * args.ny;
    g.n = g.nxy * args.nz;
    g.ix2 = args.ix2; g.iy2 = args.iy2; g.iz2 = args.iz2;
    for (int t = 0; t < 27; ++t) {
        const int mx = t / 9, my = (t / 3) % 3, mz = t % 3;
        const double dg = (2 - mx) * g.ix2 + (2 - my) * g.iy2 + (2 - mz) * g.iz2;
        g.inv_diag[t] = dg > 0.0 ? 1.0 / dg : 0.0;
        // MIXED forms z = r/diag in FP32; r.z must use the same rounded
        // Jacobi weights or the recurrences lose conjugacy.
        if (precision == FLURSYS_PRECISION_MIXED) g.inv_diag[t] = double(float(g.inv_diag[t]));
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    g.tiles_x = (g.nx + TX - 1) / TX;
    g.tiles_y = (g.ny + TY - 1) / TY;
    // Chunk length in z: about `waves` waves of four resident blocks per SM,
    // at least `kc_min` planes per chunk (FLURSYS_KC overrides both sweeps).
    const char *kc_env = std::getenv("FLURSYS_KC");
    const int kc_force = kc_env ? std::max(1, std::atoi(kc_env)) : 0;
    const long long want_tiles = (long long)sms * 4 * 2;
    auto chunking = [&](long long ncols, int *kc_out, int *chunks_out) {
        long long chunks = std::max(1LL, std::min<long long>(g.nz, want_tiles / std::max(1LL, ncols)));
        int kc = (int)((g.nz + chunks - 1) / chunks);
        kc = std::max(kc, std::min(4, g.nz));
        if (kc_force) kc = kc_force;
        kc = std::min(kc, g.nz);
        *kc_out = kc;
        *chunks_out = (g.nz + kc - 1) / kc;
    };
    chunking((long long)g.tiles_x * g.tiles_y, &g.kc, &g.chunks);
    a.nblocks_stencil = g.tiles_x * g.tiles_y * g.chunks;
    const int ryw = precision == FLURSYS_PRECISION_MIXED ? kRyOperand : kRyOperand / 2;
    g.tiles_yw = (g.ny + TY * ryw - 1) / (TY * ryw);
    chunking((long long)g.tiles_x * g.tiles_yw, &g.kcw, &g.chunksw);
    const int wv = precision == FLURSYS_PRECISION_MIXED ? 4 : 2;
    g.tiles_xv = (g.nx + 32 * wv - 1) / (32 * wv);
    g.tiles_yv = (g.ny + TY * kRyVec - 1) / (TY * kRyVec);
    chunking((long long)g.tiles_xv * g.tiles_yv, &g.kcv, &g.chunksv);
    {   // staged sweep: one wave of two blocks per SM, long chunks (the ring's
        // three extra planes are re-read per chunk)
        const long long cols = (long long)g.tiles_xv * g.tiles_yv;
        long long chunks = std::max(1LL, std::min<long long>(g.nz, (long long)sms * 2 / std::max(1LL, cols)));
        g.kcp = (int)((g.nz + chunks - 1) / chunks);
        g.chunksp = (g.nz + g.kcp - 1) / g.kcp;
    }
    // pointwise grid: 4 blocks per SM (measured on B200: 32.5 us per iteration
    // at 128^3 against 34.4 with 8, equal at 256^3); the environment variable
    // FLURSYS_PCG_POINT_BLOCKS_PER_SM overrides it
    int point_per_sm = 4;
    if (const char *env = std::getenv("FLURSYS_PCG_POINT_BLOCKS_PER_SM")) point_per_sm = std::max(1, std::atoi(env));
    a.nblocks_point = std::max(1, std::min(sms * point_per_sm, (g.n / 4 + kBlock - 1) / kBlock));
    a.x = args.x;
    a.rhs = args.rhs;
    a.r = args.r; a.d0 = args.d0; a.d1 = args.d1; a.q = args.q; a.dx = args.dx;
    a.row_class = args.row_class;
    a.stop_rule = args.stop_rule;
    a.tol = args.tol; a.atol = args.atol; a.rtol = args.rtol;
    a.max_iters = args.max_iters;
    a.replace_every = args.replace_every > 0 ? args.replace_every : 50;
    const int nb = std::max({a.nblocks_stencil, a.nblocks_point, g.tiles_x * g.tiles_yw * g.chunksw,
                             g.tiles_xv * g.tiles_yv * g.chunksv, g.tiles_xv * g.tiles_yv * g.chunksp,
                             g.tiles_x * g.tiles_y * ((g.nz + 3) / 4)});
    cudaError_t e = cudaMalloc(&plan.partials, sizeof(double) * kSlots * nb);
    if (e == cudaSuccess) e = cudaMalloc(&plan.state, sizeof(CgSeqState));
    if (e == cudaSuccess) e = cudaMemset(plan.state, 0, sizeof(CgSeqState));
    if (e != cudaSuccess) return e;
    a.partials = plan.partials;
    a.st = plan.state;
    plan.precision = precision;
    a.graph = 1;
    const char *st = std::getenv("FLURSYS_STENCIL");
    const bool vec_ok = g.nx % wv == 0;
    // MIXED takes the staged sweep (FLURSYS_STENCIL=vec selects the register
    // sweep); FP64 the register sweep
    a.sweep = vec_ok ? (precision == FLURSYS_PRECISION_MIXED ? kSweepPipe : kSweepVec) : kSweepTile;
    if (st && std::strcmp(st, "vec") == 0 && vec_ok) a.sweep = kSweepVec;
    if (st && std::strcmp(st, "direct") == 0) a.sweep = kSweepDirect;
    if (st && std::strcmp(st, "tiled") == 0) a.sweep = kSweepTile;
    if (st && std::strcmp(st, "warp") == 0) a.sweep = kSweepWarp;
    a.nblocks_dir = a.sweep == kSweepWarp ? g.tiles_x * g.tiles_yw * g.chunksw
                  : a.sweep == kSweepVec  ? g.tiles_xv * g.tiles_yv * g.chunksv
                  : a.sweep == kSweepPipe ? g.tiles_xv * g.tiles_yv * g.chunksp
                                          : a.nblocks_stencil;
    if (a.sweep == kSweepPipe) {
        e = cudaFuncSetAttribute((const void *)seq_dir_pipe, cudaFuncAttributeMaxDynamicSharedMemorySize, kPipeSmem);
        if (e != cudaSuccess) return e;
    }
    // FLURSYS_PCG_CG1=1 selects the single-reduction variant for MIXED when
    // the TMA maps can be made (nx % 4 == 0); FLURSYS_CG1_TZ=4 selects
    // 4-plane tiles (8 by default). It is not the default: on B200 at 128^3
    // it takes 39.5 us per iteration against 32.5 us for the two-launch form
    // (instruction-bound by the halo recomputation, 238 instructions per cell).
    const char *cg1_env = std::getenv("FLURSYS_PCG_CG1");
    a.cg1 = precision == FLURSYS_PRECISION_MIXED && g.nx % 4 == 0 && cg1_env && std::strcmp(cg1_env, "1") == 0;
    Cg1Maps maps{};
    if (a.cg1) {
        a.cr[0] = static_cast<float *>(args.r);
        a.cr[1] = static_cast<float *>(args.q);
        a.cp[0] = static_cast<float *>(args.d0);
        a.cp[1] = static_cast<float *>(args.d1);
        const char *tz_env = std::getenv("FLURSYS_CG1_TZ");
        a.cg1_tz = tz_env && std::atoi(tz_env) == 4 ? 4 : 8;
        const unsigned tz = (unsigned)a.cg1_tz;
        bool ok = true;
        for (int b = 0; b < 2; ++b) {
            ok = ok && tma_map_f32_3d(&maps.r[b], a.cr[b], g.nx, g.ny, g.nz, TX + 8, TY + 4, tz + 4);
            ok = ok && tma_map_f32_3d(&maps.p[b], a.cp[b], g.nx, g.ny, g.nz, TX + 8, TY + 4, tz + 4);
        }
        ok = ok && tma_map_f32_3d(&maps.dx, args.dx, g.nx, g.ny, g.nz, TX, TY, tz);
        if (!ok) return cudaErrorNotSupported;
        a.nblocks_cg1 = g.tiles_x * g.tiles_y * ((g.nz + a.cg1_tz - 1) / a.cg1_tz);
        const void *fn = a.cg1_tz == 4 ? (const void *)cg1_tile<4> : (const void *)cg1_tile<8>;
        const int smem = (int)(a.cg1_tz == 4 ? Cg1Tile<4>::smem_bytes : Cg1Tile<8>::smem_bytes);
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        plan.cg1_maps = new Cg1Maps(maps);
        e = build_cg1(plan, a, maps);
    } else {
        e = precision == FLURSYS_PRECISION_MIXED ? build<float, true>(plan, a) : build<double, false>(plan, a);
    }
    plan.host_args = new SeqArgs(a);
    const char *v = std::getenv("FLURSYS_PCG_VARIANT");
    if (v && std::strcmp(v, "host") == 0) plan.host_iterations = 1;
    // MIXED solves whose tiles fit one per SM run chip-resident (one
    // cooperative launch per solve; FLURSYS_PCG_RESIDENT=0 keeps the graph).
    if (e == cudaSuccess && precision == FLURSYS_PRECISION_MIXED && !a.cg1 && plan.host_iterations == 0) {
        auto *rp = new Pcg3dResPlan();
        if (pcg3d_res_plan(*rp, args, device)) plan.resident = rp;
        else delete rp;
        cudaGetLastError();  // a declined plan leaves no sticky error behind
    }
    return e;
}

cudaError_t pcg3d_seq_launch(const Pcg3dSeqPlan &plan, cudaStream_t stream) {
    if (plan.resident) return pcg3d_res_launch(*plan.resident, plan.state, stream);
    if (plan.host_iterations > 0) return pcg3d_seq_run_host(plan, stream);
    return cudaGraphLaunch(plan.exec, stream);
}

// Host-driven mode (diagnostics): the same kernels launched one by one from
// the host, so profilers that cannot look inside conditional graph nodes see
// every launch. The kernels honour the device flags (`done`, `replace`)
// exactly as the graph's conditional nodes do; the host checks `done` after
// every chunk of 16 iterations.
cudaError_t pcg3d_seq_run_host(const Pcg3dSeqPlan &plan, cudaStream_t st) {
    SeqArgs a = *static_cast<const SeqArgs *>(plan.host_args);
    a.graph = 0;
    const bool mixed = plan.precision == FLURSYS_PRECISION_MIXED;
    if (a.cg1) {
        seq_init<float, true><<<a.nblocks_stencil, kBlock, 0, st>>>(a);
        cg1_ws<0><<<a.nblocks_stencil, kBlock, 0, st>>>(a);
        int done = 0;
        for (long long it = 0; it < a.max_iters && !done; it += 16) {
            for (int j = 0; j < 16; ++j) {
                const Cg1Maps &maps = *static_cast<const Cg1Maps *>(plan.cg1_maps);
                if (a.cg1_tz == 4) cg1_tile<4><<<a.nblocks_cg1, kBlock, Cg1Tile<4>::smem_bytes, st>>>(a, maps);
                else cg1_tile<8><<<a.nblocks_cg1, kBlock, Cg1Tile<8>::smem_bytes, st>>>(a, maps);
                seq_fold<<<a.nblocks_point, kBlock, 0, st>>>(a);
                cg1_replace_r<<<a.nblocks_stencil, kBlock, 0, st>>>(a);
                cg1_ws<1><<<a.nblocks_stencil, kBlock, 0, st>>>(a);
            }
            cudaError_t e = cudaMemcpyAsync(&done, &plan.state->done, sizeof(int), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return e;
        }
        seq_fold_pending<<<a.nblocks_point, kBlock, 0, st>>>(a);
        seq_final<float, true><<<a.nblocks_stencil, kBlock, 0, st>>>(a);
        return cudaGetLastError();
    }
    if (mixed) seq_init<float, true><<<a.nblocks_stencil, kBlock, 0, st>>>(a);
    else seq_init<double, false><<<a.nblocks_stencil, kBlock, 0, st>>>(a);
    int done = 0;
    for (long long it = 0; it < a.max_iters && !done; it += 16) {
        for (int j = 0; j < 16; ++j) {
            if (mixed) {
                if (a.sweep == kSweepVec) seq_dir_vec<float, true, kRyVec><<<a.nblocks_dir, kBlock, 0, st>>>(a);
                else if (a.sweep == kSweepPipe) seq_dir_pipe<<<a.nblocks_dir, kBlock, kPipeSmem, st>>>(a);
                else seq_dir_spmv<float, true><<<a.nblocks_dir, kBlock, 0, st>>>(a);
                seq_update<float, true><<<a.nblocks_point, kBlock, 0, st>>>(a);
                seq_fold<<<a.nblocks_point, kBlock, 0, st>>>(a);
                seq_replace<float, true><<<a.nblocks_stencil, kBlock, 0, st>>>(a);
            } else {
                if (a.sweep == kSweepVec) seq_dir_vec<double, false, kRyVec><<<a.nblocks_dir, kBlock, 0, st>>>(a);
                else seq_dir_spmv<double, false><<<a.nblocks_dir, kBlock, 0, st>>>(a);
                seq_update<double, false><<<a.nblocks_point, kBlock, 0, st>>>(a);
            }
        }
        cudaError_t e = cudaMemcpyAsync(&done, &plan.state->done, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return e;
    }
    if (mixed) {
        seq_fold_pending<<<a.nblocks_point, kBlock, 0, st>>>(a);
        seq_final<float, true><<<a.nblocks_stencil, kBlock, 0, st>>>(a);
    } else {
        seq_final<double, false><<<a.nblocks_stencil, kBlock, 0, st>>>(a);
    }
    return cudaGetLastError();
}

void pcg3d_seq_destroy(Pcg3dSeqPlan &plan) {
    if (plan.resident) {
        pcg3d_res_destroy(*plan.resident);
        delete plan.resident;
    }
    delete static_cast<SeqArgs *>(plan.host_args);
    if (plan.exec) cudaGraphExecDestroy(plan.exec);
    if (plan.graph) cudaGraphDestroy(plan.graph);
    cudaFree(plan.partials);
    cudaFree(plan.state);
    delete static_cast<Cg1Maps *>(plan.cg1_maps);
    plan = Pcg3dSeqPlan{};
}

}  // namespace flursys
