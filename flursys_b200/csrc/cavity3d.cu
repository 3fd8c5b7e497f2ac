// cavity3d.cu — velocity phases of the 3D lid-driven-cavity projection step
// (src/solver/incompressible_3d.rs) on sm_100a, all in FP64.
//
// Layout (Field3D, src/field.rs:104): x fastest, idx = i + nx*(j + ny*k);
// u is (nx+1) x ny x nz, v is nx x (ny+1) x nz, w is nx x ny x (nz+1).
// Every kernel writes each output element exactly once (the zero fill of the
// reference's predictor is folded into the predictor kernels).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "cavity3d.cuh"
#include "common.cuh"

namespace flursys {

namespace {

constexpr int kRowBlk = 128;  // threads along x of the row-mapped kernels

// Grid spacings and their reciprocals (the kernels multiply by these in
// place of the reference's divisions by 2 h, h^2 and h).
struct G3 {
    int nx, ny, nz;
    double dx, dy, dz;
    double i2dx, i2dy, i2dz;  // 1 / (2 h)
    double idx2, idy2, idz2;  // 1 / h^2
    double idx, idy, idz;     // 1 / h
};

G3 make_g3(int nx, int ny, int nz, double dx, double dy, double dz) {
    return G3{nx, ny, nz, dx, dy, dz, 1.0 / (2.0 * dx), 1.0 / (2.0 * dy), 1.0 / (2.0 * dz),
              1.0 / (dx * dx), 1.0 / (dy * dy), 1.0 / (dz * dz), 1.0 / dx, 1.0 / dy, 1.0 / dz};
}

// Row mapping of the face / cell kernels: one block row of x per (j, k)
// (blockIdx.y = j, blockIdx.z = k), no index division.
dim3 row_grid(long long sx, int sy, int sz) { return dim3((unsigned)((sx + kRowBlk - 1) / kRowBlk), sy, sz); }

// predict_momentum, u component (incompressible_3d.rs:181-210).
__global__ void __launch_bounds__(kRowBlk) predict_u(const double *__restrict__ u, const double *__restrict__ v,
                                                     const double *__restrict__ w, double *__restrict__ us,
                                                     G3 g, double dt, double nu, double lid) {
    // threads cover i < nx (whole blocks for nx a multiple of 128); the
    // thread of i = 0 also writes the wall face i = nx
    const int i = blockIdx.x * kRowBlk + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    const long long sx = g.nx + 1;
    if (i >= g.nx) return;
    const long long id = i + sx * (j + (long long)g.ny * k);
    if (i == 0) {
        us[id] = 0.0;
        us[id + g.nx] = 0.0;
        return;
    }
    const double c = __ldg(u + id);
    const double e = __ldg(u + id + 1), wst = __ldg(u + id - 1);
    // u_neighbor (incompressible_3d.rs:365-393): ghost 2 lid - c above the
    // top wall, -c at the other walls
    const long long suz = sx * g.ny;
    const double nn = (j + 1 < g.ny) ? __ldg(u + id + sx) : 2.0 * lid - c;
    const double s = (j > 0) ? __ldg(u + id - sx) : -c;
    const double f = (k + 1 < g.nz) ? __ldg(u + id + suz) : -c;
    const double b = (k > 0) ? __ldg(u + id - suz) : -c;
    const long long sv = g.nx, svz = (long long)g.nx * (g.ny + 1);
    const double vb = 0.25 * (__ldg(v + (i - 1) + sv * j + svz * k) + __ldg(v + i + sv * j + svz * k) +
                              __ldg(v + (i - 1) + sv * (j + 1) + svz * k) + __ldg(v + i + sv * (j + 1) + svz * k));
    const long long sw = g.nx, swz = (long long)g.nx * g.ny;
    const double wb = 0.25 * (__ldg(w + (i - 1) + sw * j + swz * k) + __ldg(w + i + sw * j + swz * k) +
                              __ldg(w + (i - 1) + sw * j + swz * (k + 1)) + __ldg(w + i + sw * j + swz * (k + 1)));
    us[id] = c + dt * (-c * (e - wst) * g.i2dx - vb * (nn - s) * g.i2dy - wb * (f - b) * g.i2dz +
                       nu * ((e - 2.0 * c + wst) * g.idx2 + (nn - 2.0 * c + s) * g.idy2 + (f - 2.0 * c + b) * g.idz2));
}

// predict_momentum, v component (incompressible_3d.rs:212-241); v_neighbor :395-420.
__global__ void __launch_bounds__(kRowBlk) predict_v(const double *__restrict__ u, const double *__restrict__ v,
                                                     const double *__restrict__ w, double *__restrict__ vs,
                                                     G3 g, double dt, double nu) {
    const int i = blockIdx.x * kRowBlk + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    const long long sx = g.nx, sz = (long long)g.nx * (g.ny + 1);
    if (i >= sx) return;
    const long long id = i + sx * (j + (long long)(g.ny + 1) * k);
    if (j == 0 || j == g.ny) { vs[id] = 0.0; return; }
    const double c = __ldg(v + id);
    const double e = (i + 1 < g.nx) ? __ldg(v + id + 1) : -c;
    const double wst = (i > 0) ? __ldg(v + id - 1) : -c;
    const double nn = __ldg(v + id + sx), s = __ldg(v + id - sx);
    const double f = (k + 1 < g.nz) ? __ldg(v + id + sz) : -c;
    const double b = (k > 0) ? __ldg(v + id - sz) : -c;
    const long long su = g.nx + 1, suz = (long long)(g.nx + 1) * g.ny;
    const double ub = 0.25 * (__ldg(u + i + su * (j - 1) + suz * k) + __ldg(u + (i + 1) + su * (j - 1) + suz * k) +
                              __ldg(u + i + su * j + suz * k) + __ldg(u + (i + 1) + su * j + suz * k));
    const long long sw = g.nx, swz = (long long)g.nx * g.ny;
    const double wb = 0.25 * (__ldg(w + i + sw * (j - 1) + swz * k) + __ldg(w + i + sw * j + swz * k) +
                              __ldg(w + i + sw * (j - 1) + swz * (k + 1)) + __ldg(w + i + sw * j + swz * (k + 1)));
    vs[id] = c + dt * (-ub * (e - wst) * g.i2dx - c * (nn - s) * g.i2dy - wb * (f - b) * g.i2dz +
                       nu * ((e - 2.0 * c + wst) * g.idx2 + (nn - 2.0 * c + s) * g.idy2 + (f - 2.0 * c + b) * g.idz2));
}

// predict_momentum, w component (incompressible_3d.rs:243-272); w_neighbor :422-447.
__global__ void __launch_bounds__(kRowBlk) predict_w(const double *__restrict__ u, const double *__restrict__ v,
                                                     const double *__restrict__ w, double *__restrict__ ws,
                                                     G3 g, double dt, double nu) {
    const int i = blockIdx.x * kRowBlk + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    const long long sx = g.nx, sz = (long long)g.nx * g.ny;
    if (i >= sx) return;
    const long long id = i + sx * (j + (long long)g.ny * k);
    if (k == 0 || k == g.nz) { ws[id] = 0.0; return; }
    const double c = __ldg(w + id);
    const double e = (i + 1 < g.nx) ? __ldg(w + id + 1) : -c;
    const double wst = (i > 0) ? __ldg(w + id - 1) : -c;
    const double nn = (j + 1 < g.ny) ? __ldg(w + id + sx) : -c;
    const double s = (j > 0) ? __ldg(w + id - sx) : -c;
    const double f = __ldg(w + id + sz), b = __ldg(w + id - sz);
    const long long su = g.nx + 1, suz = (long long)(g.nx + 1) * g.ny;
    const double ub = 0.25 * (__ldg(u + i + su * j + suz * (k - 1)) + __ldg(u + (i + 1) + su * j + suz * (k - 1)) +
                              __ldg(u + i + su * j + suz * k) + __ldg(u + (i + 1) + su * j + suz * k));
    const long long sv = g.nx, svz = (long long)g.nx * (g.ny + 1);
    const double vb = 0.25 * (__ldg(v + i + sv * j + svz * (k - 1)) + __ldg(v + i + sv * (j + 1) + svz * (k - 1)) +
                              __ldg(v + i + sv * j + svz * k) + __ldg(v + i + sv * (j + 1) + svz * k));
    ws[id] = c + dt * (-ub * (e - wst) * g.i2dx - vb * (nn - s) * g.i2dy - c * (f - b) * g.i2dz +
                       nu * ((e - 2.0 * c + wst) * g.idx2 + (nn - 2.0 * c + s) * g.idy2 + (f - 2.0 * c + b) * g.idz2));
}

// build_pressure_rhs (incompressible_3d.rs:275-291), rhs(0,0,0) = 0.
__global__ void __launch_bounds__(kRowBlk) build_rhs(const double *__restrict__ us, const double *__restrict__ vs,
                                                     const double *__restrict__ ws, double *__restrict__ rhs, G3 g,
                                                     double scale) {
    const int i = blockIdx.x * kRowBlk + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= g.nx) return;
    const long long id = i + (long long)g.nx * (j + (long long)g.ny * k);
    if (id == 0) { rhs[0] = 0.0; return; }
    const long long iu = i + (long long)(g.nx + 1) * (j + (long long)g.ny * k);
    const long long iv = i + (long long)g.nx * (j + (long long)(g.ny + 1) * k);
    rhs[id] = scale * (__ldg(us + iu + 1) - __ldg(us + iu)) * g.idx +
              scale * (__ldg(vs + iv + g.nx) - __ldg(vs + iv)) * g.idy +
              scale * (__ldg(ws + id + (long long)g.nx * g.ny) - __ldg(ws + id)) * g.idz;
}

// correct_velocity (incompressible_3d.rs:334-363): interior faces only.
__global__ void __launch_bounds__(kRowBlk) correct_all(const double *__restrict__ us, const double *__restrict__ vs,
                                                       const double *__restrict__ ws, const double *__restrict__ p,
                                                       double *__restrict__ u, double *__restrict__ v,
                                                       double *__restrict__ w, G3 g, double scale) {
    const int i = blockIdx.x * kRowBlk + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= g.nx) return;
    const long long sxy = (long long)g.nx * g.ny;
    const long long id = i + (long long)g.nx * (j + (long long)g.ny * k);
    const double pc = __ldg(p + id);
    if (i > 0) {
        const long long iu = i + (long long)(g.nx + 1) * (j + (long long)g.ny * k);
        u[iu] = __ldg(us + iu) - scale * (pc - __ldg(p + id - 1)) * g.idx;
    }
    if (j > 0) {
        const long long iv = i + (long long)g.nx * (j + (long long)(g.ny + 1) * k);
        v[iv] = __ldg(vs + iv) - scale * (pc - __ldg(p + id - g.nx)) * g.idy;
    }
    if (k > 0) w[id] = __ldg(ws + id) - scale * (pc - __ldg(p + id - sxy)) * g.idz;
}

__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v) {
    // Non-negative doubles order like their bit patterns.
    atomicMax(reinterpret_cast<unsigned long long *>(addr), __double_as_longlong(v));
}

// max_divergence (:504-517), max_speed (:519-532) and the ensure_finite scan
// (:534-554) of p, u, v, w in one pass. Blocks stride over the rows (j, k) of
// the (nx+1) x (ny+1) x (nz+1) index box with their threads along x, so a
// thread never divides an index; one block maximum per block goes to the
// result.
__global__ void __launch_bounds__(kRowBlk) diagnostics(const double *__restrict__ u, const double *__restrict__ v,
                                                    const double *__restrict__ w, const double *__restrict__ p,
                                                    G3 g, Diag3Dev *out) {
    __shared__ double s_red[kRowBlk / 32];
    const int rows = (g.ny + 1) * (g.nz + 1);
    double mdiv = 0.0, mspeed2 = 0.0;  // the speed's maximum is taken squared; sqrt is monotone
    for (int row = blockIdx.x; row < rows; row += gridDim.x) {
        const int k = row / (g.ny + 1), j = row - k * (g.ny + 1);
        const bool yin = j < g.ny, zin = k < g.nz;
        if (threadIdx.x == 0 && yin && zin) {  // the u face i = nx of this row
            const long long iu = g.nx + (long long)(g.nx + 1) * (j + (long long)g.ny * k);
            if (!isfinite(__ldg(u + iu))) atomicMin(&out->bad_index[1], (unsigned long long)iu);
        }
        for (int i = threadIdx.x; i < g.nx; i += kRowBlk) {
            if (yin && zin) {
                const long long id = i + (long long)g.nx * (j + (long long)g.ny * k);
                const long long iu = i + (long long)(g.nx + 1) * (j + (long long)g.ny * k);
                const long long iv = i + (long long)g.nx * (j + (long long)(g.ny + 1) * k);
                const double u0 = __ldg(u + iu), u1 = __ldg(u + iu + 1);
                const double v0 = __ldg(v + iv), v1 = __ldg(v + iv + g.nx);
                const double w0 = __ldg(w + id), w1 = __ldg(w + id + (long long)g.nx * g.ny);
                const double div = (u1 - u0) * g.idx + (v1 - v0) * g.idy + (w1 - w0) * g.idz;
                mdiv = fmax(mdiv, fabs(div));
                const double a = 0.5 * (u0 + u1), b = 0.5 * (v0 + v1), c = 0.5 * (w0 + w1);
                mspeed2 = fmax(mspeed2, a * a + b * b + c * c);
                if (!isfinite(__ldg(p + id))) atomicMin(&out->bad_index[0], (unsigned long long)id);
            }
            if (yin && zin) {  // u face (i, j, k), i < nx
                const long long iu = i + (long long)(g.nx + 1) * (j + (long long)g.ny * k);
                if (!isfinite(__ldg(u + iu))) atomicMin(&out->bad_index[1], (unsigned long long)iu);
            }
            if (zin) {  // v face, j <= ny
                const long long iv = i + (long long)g.nx * (j + (long long)(g.ny + 1) * k);
                if (!isfinite(__ldg(v + iv))) atomicMin(&out->bad_index[2], (unsigned long long)iv);
            }
            if (yin) {  // w face, k <= nz
                const long long iw = i + (long long)g.nx * (j + (long long)g.ny * k);
                if (!isfinite(__ldg(w + iw))) atomicMin(&out->bad_index[3], (unsigned long long)iw);
            }
        }
    }
    const double bd = block_max<kRowBlk>(mdiv, s_red);
    const double bs = sqrt(block_max<kRowBlk>(mspeed2, s_red));
    if (threadIdx.x == 0) {
        atomic_max_nonneg(&out->max_divergence, bd);
        atomic_max_nonneg(&out->max_speed, bs);
    }
}

__global__ void diag_reset(Diag3Dev *out) {
    out->max_divergence = 0.0;
    out->max_speed = 0.0;
    for (int f = 0; f < 4; ++f) out->bad_index[f] = ~0ull;
}

}  // namespace

cudaError_t cavity3d_predict(const Cavity3dState &s, double dt, cudaStream_t st) {
    const G3 g = make_g3(s.nx, s.ny, s.nz, s.dx, s.dy, s.dz);
    predict_u<<<row_grid(s.nx, s.ny, s.nz), kRowBlk, 0, st>>>(s.u, s.v, s.w, s.us, g, dt, s.nu, s.lid);
    predict_v<<<row_grid(s.nx, s.ny + 1, s.nz), kRowBlk, 0, st>>>(s.u, s.v, s.w, s.vs, g, dt, s.nu);
    predict_w<<<row_grid(s.nx, s.ny, s.nz + 1), kRowBlk, 0, st>>>(s.u, s.v, s.w, s.ws, g, dt, s.nu);
    return cudaGetLastError();
}

cudaError_t cavity3d_rhs(const Cavity3dState &s, double dt, cudaStream_t st) {
    const G3 g = make_g3(s.nx, s.ny, s.nz, s.dx, s.dy, s.dz);
    build_rhs<<<row_grid(s.nx, s.ny, s.nz), kRowBlk, 0, st>>>(s.us, s.vs, s.ws, s.rhs, g, s.rho / dt);
    return cudaGetLastError();
}

cudaError_t cavity3d_correct(const Cavity3dState &s, double dt, cudaStream_t st) {
    const G3 g = make_g3(s.nx, s.ny, s.nz, s.dx, s.dy, s.dz);
    correct_all<<<row_grid(s.nx, s.ny, s.nz), kRowBlk, 0, st>>>(s.us, s.vs, s.ws, s.p, s.u, s.v, s.w, g, dt / s.rho);
    return cudaGetLastError();
}

cudaError_t cavity3d_diagnostics(const Cavity3dState &s, Diag3Dev *out, cudaStream_t st) {
    const G3 g = make_g3(s.nx, s.ny, s.nz, s.dx, s.dy, s.dz);
    diag_reset<<<1, 1, 0, st>>>(out);
    const long long rows = (long long)(s.ny + 1) * (s.nz + 1);
    const int blocks = (int)std::min<long long>(rows, (long long)s.sms * 16);
    diagnostics<<<blocks, kRowBlk, 0, st>>>(s.u, s.v, s.w, s.p, g, out);
    return cudaGetLastError();
}

}  // namespace flursys
