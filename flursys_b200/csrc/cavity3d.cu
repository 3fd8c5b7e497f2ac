// cavity3d.cu — velocity phases of the 3D lid-driven-cavity projection step
// (src/solver/incompressible_3d.rs) on sm_100a, all in FP64.
//
// Layout (Field3D, src/field.rs:104): x fastest, idx = i + nx*(j + ny*k);
// u is (nx+1) x ny x nz, v is nx x (ny+1) x nz, w is nx x ny x (nz+1).
// Every kernel writes each output element exactly once (the zero fill of the
// reference's predictor is folded into the predictor kernels).
#include <cuda_runtime.h>

#include <cmath>

#include "cavity3d.cuh"
#include "common.cuh"

namespace flursys {

namespace {

constexpr int kBlk = 256;

struct G3 {
    int nx, ny, nz;
    double dx, dy, dz;
};

// u_neighbor (incompressible_3d.rs:365-393) for an interior u face.
__device__ __forceinline__ double unb(const double *__restrict__ u, const G3 &g, int i, int j, int k,
                                      int dj, int dk, double c, double lid) {
    const int nj = j + dj, nk = k + dk;
    if (nj >= 0 && nj < g.ny && nk >= 0 && nk < g.nz)
        return __ldg(u + i + (long long)(g.nx + 1) * (nj + (long long)g.ny * nk));
    return nj >= g.ny ? 2.0 * lid - c : -c;
}

// predict_momentum, u component (incompressible_3d.rs:181-210).
__global__ void __launch_bounds__(kBlk) predict_u(const double *__restrict__ u, const double *__restrict__ v,
                                                  const double *__restrict__ w, double *__restrict__ us,
                                                  G3 g, double dt, double nu, double lid) {
    const long long n = (long long)(g.nx + 1) * g.ny * g.nz;
    const long long sx = g.nx + 1;
    for (long long id = (long long)blockIdx.x * kBlk + threadIdx.x; id < n; id += (long long)gridDim.x * kBlk) {
        const int i = int(id % sx);
        const long long jk = id / sx;
        const int j = int(jk % g.ny), k = int(jk / g.ny);
        if (i == 0 || i == g.nx) { us[id] = 0.0; continue; }
        const double c = __ldg(u + id);
        const double e = __ldg(u + id + 1), wst = __ldg(u + id - 1);
        const double nn = unb(u, g, i, j, k, 1, 0, c, lid), s = unb(u, g, i, j, k, -1, 0, c, lid);
        const double f = unb(u, g, i, j, k, 0, 1, c, lid), b = unb(u, g, i, j, k, 0, -1, c, lid);
        const long long sv = g.nx, svz = (long long)g.nx * (g.ny + 1);
        const double vb = 0.25 * (__ldg(v + (i - 1) + sv * j + svz * k) + __ldg(v + i + sv * j + svz * k) +
                                  __ldg(v + (i - 1) + sv * (j + 1) + svz * k) + __ldg(v + i + sv * (j + 1) + svz * k));
        const long long sw = g.nx, swz = (long long)g.nx * g.ny;
        const double wb = 0.25 * (__ldg(w + (i - 1) + sw * j + swz * k) + __ldg(w + i + sw * j + swz * k) +
                                  __ldg(w + (i - 1) + sw * j + swz * (k + 1)) + __ldg(w + i + sw * j + swz * (k + 1)));
        us[id] = c + dt * (-c * (e - wst) / (2.0 * g.dx) - vb * (nn - s) / (2.0 * g.dy) - wb * (f - b) / (2.0 * g.dz) +
                           nu * ((e - 2.0 * c + wst) / (g.dx * g.dx) + (nn - 2.0 * c + s) / (g.dy * g.dy) +
                                 (f - 2.0 * c + b) / (g.dz * g.dz)));
    }
}

// predict_momentum, v component (incompressible_3d.rs:212-241); v_neighbor :395-420.
__global__ void __launch_bounds__(kBlk) predict_v(const double *__restrict__ u, const double *__restrict__ v,
                                                  const double *__restrict__ w, double *__restrict__ vs,
                                                  G3 g, double dt, double nu) {
    const long long n = (long long)g.nx * (g.ny + 1) * g.nz;
    const long long sx = g.nx, sz = (long long)g.nx * (g.ny + 1);
    for (long long id = (long long)blockIdx.x * kBlk + threadIdx.x; id < n; id += (long long)gridDim.x * kBlk) {
        const int i = int(id % sx);
        const long long jk = id / sx;
        const int j = int(jk % (g.ny + 1)), k = int(jk / (g.ny + 1));
        if (j == 0 || j == g.ny) { vs[id] = 0.0; continue; }
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
        vs[id] = c + dt * (-ub * (e - wst) / (2.0 * g.dx) - c * (nn - s) / (2.0 * g.dy) - wb * (f - b) / (2.0 * g.dz) +
                           nu * ((e - 2.0 * c + wst) / (g.dx * g.dx) + (nn - 2.0 * c + s) / (g.dy * g.dy) +
                                 (f - 2.0 * c + b) / (g.dz * g.dz)));
    }
}

// predict_momentum, w component (incompressible_3d.rs:243-272); w_neighbor :422-447.
__global__ void __launch_bounds__(kBlk) predict_w(const double *__restrict__ u, const double *__restrict__ v,
                                                  const double *__restrict__ w, double *__restrict__ ws,
                                                  G3 g, double dt, double nu) {
    const long long n = (long long)g.nx * g.ny * (g.nz + 1);
    const long long sx = g.nx, sz = (long long)g.nx * g.ny;
    for (long long id = (long long)blockIdx.x * kBlk + threadIdx.x; id < n; id += (long long)gridDim.x * kBlk) {
        const int i = int(id % sx);
        const long long jk = id / sx;
        const int j = int(jk % g.ny), k = int(jk / g.ny);
        if (k == 0 || k == g.nz) { ws[id] = 0.0; continue; }
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
        ws[id] = c + dt * (-ub * (e - wst) / (2.0 * g.dx) - vb * (nn - s) / (2.0 * g.dy) - c * (f - b) / (2.0 * g.dz) +
                           nu * ((e - 2.0 * c + wst) / (g.dx * g.dx) + (nn - 2.0 * c + s) / (g.dy * g.dy) +
                                 (f - 2.0 * c + b) / (g.dz * g.dz)));
    }
}

// build_pressure_rhs (incompressible_3d.rs:275-291), rhs(0,0,0) = 0.
__global__ void __launch_bounds__(kBlk) build_rhs(const double *__restrict__ us, const double *__restrict__ vs,
                                                  const double *__restrict__ ws, double *__restrict__ rhs, G3 g,
                                                  double scale) {
    const long long n = (long long)g.nx * g.ny * g.nz;
    for (long long id = (long long)blockIdx.x * kBlk + threadIdx.x; id < n; id += (long long)gridDim.x * kBlk) {
        const int i = int(id % g.nx);
        const long long jk = id / g.nx;
        const int j = int(jk % g.ny), k = int(jk / g.ny);
        if (id == 0) { rhs[0] = 0.0; continue; }
        const long long iu = i + (long long)(g.nx + 1) * (j + (long long)g.ny * k);
        const long long iv = i + (long long)g.nx * (j + (long long)(g.ny + 1) * k);
        rhs[id] = scale * (__ldg(us + iu + 1) - __ldg(us + iu)) / g.dx +
                  scale * (__ldg(vs + iv + g.nx) - __ldg(vs + iv)) / g.dy +
                  scale * (__ldg(ws + id + (long long)g.nx * g.ny) - __ldg(ws + id)) / g.dz;
    }
}

// correct_velocity (incompressible_3d.rs:334-363): interior faces only.
__global__ void __launch_bounds__(kBlk) correct_all(const double *__restrict__ us, const double *__restrict__ vs,
                                                    const double *__restrict__ ws, const double *__restrict__ p,
                                                    double *__restrict__ u, double *__restrict__ v,
                                                    double *__restrict__ w, G3 g, double scale) {
    const long long n = (long long)g.nx * g.ny * g.nz;
    const long long sxy = (long long)g.nx * g.ny;
    for (long long id = (long long)blockIdx.x * kBlk + threadIdx.x; id < n; id += (long long)gridDim.x * kBlk) {
        const int i = int(id % g.nx);
        const long long jk = id / g.nx;
        const int j = int(jk % g.ny), k = int(jk / g.ny);
        const double pc = __ldg(p + id);
        if (i > 0) {
            const long long iu = i + (long long)(g.nx + 1) * (j + (long long)g.ny * k);
            u[iu] = __ldg(us + iu) - scale * (pc - __ldg(p + id - 1)) / g.dx;
        }
        if (j > 0) {
            const long long iv = i + (long long)g.nx * (j + (long long)(g.ny + 1) * k);
            v[iv] = __ldg(vs + iv) - scale * (pc - __ldg(p + id - g.nx)) / g.dy;
        }
        if (k > 0) w[id] = __ldg(ws + id) - scale * (pc - __ldg(p + id - sxy)) / g.dz;
    }
}

__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v) {
    // Non-negative doubles order like their bit patterns.
    atomicMax(reinterpret_cast<unsigned long long *>(addr), __double_as_longlong(v));
}

// max_divergence (:504-517), max_speed (:519-532) and the ensure_finite scan
// (:534-554) of p, u, v, w in one pass.
__global__ void __launch_bounds__(kBlk) diagnostics(const double *__restrict__ u, const double *__restrict__ v,
                                                    const double *__restrict__ w, const double *__restrict__ p,
                                                    G3 g, Diag3Dev *out) {
    __shared__ double s_red[kBlk / 32];
    const long long nc = (long long)g.nx * g.ny * g.nz;
    const long long nu_ = (long long)(g.nx + 1) * g.ny * g.nz;
    const long long nv_ = (long long)g.nx * (g.ny + 1) * g.nz;
    const long long nw_ = (long long)g.nx * g.ny * (g.nz + 1);
    const long long nmax = nu_ > nv_ ? (nu_ > nw_ ? nu_ : nw_) : (nv_ > nw_ ? nv_ : nw_);
    double mdiv = 0.0, mspeed = 0.0;
    for (long long id = (long long)blockIdx.x * kBlk + threadIdx.x; id < nmax; id += (long long)gridDim.x * kBlk) {
        if (id < nc) {
            const int i = int(id % g.nx);
            const long long jk = id / g.nx;
            const int j = int(jk % g.ny), k = int(jk / g.ny);
            const long long iu = i + (long long)(g.nx + 1) * (j + (long long)g.ny * k);
            const long long iv = i + (long long)g.nx * (j + (long long)(g.ny + 1) * k);
            const double u0 = __ldg(u + iu), u1 = __ldg(u + iu + 1);
            const double v0 = __ldg(v + iv), v1 = __ldg(v + iv + g.nx);
            const double w0 = __ldg(w + id), w1 = __ldg(w + id + (long long)g.nx * g.ny);
            const double div = (u1 - u0) / g.dx + (v1 - v0) / g.dy + (w1 - w0) / g.dz;
            mdiv = fmax(mdiv, fabs(div));
            const double a = 0.5 * (u0 + u1), b = 0.5 * (v0 + v1), c = 0.5 * (w0 + w1);
            mspeed = fmax(mspeed, sqrt(a * a + b * b + c * c));
            if (!isfinite(__ldg(p + id))) atomicMin(&out->bad_index[0], (unsigned long long)id);
        }
        if (id < nu_ && !isfinite(__ldg(u + id))) atomicMin(&out->bad_index[1], (unsigned long long)id);
        if (id < nv_ && !isfinite(__ldg(v + id))) atomicMin(&out->bad_index[2], (unsigned long long)id);
        if (id < nw_ && !isfinite(__ldg(w + id))) atomicMin(&out->bad_index[3], (unsigned long long)id);
    }
    const double bd = block_max<kBlk>(mdiv, s_red);
    const double bs = block_max<kBlk>(mspeed, s_red);
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

int grid_for(long long n, int sms) {
    long long b = (n + kBlk - 1) / kBlk;
    long long cap = (long long)sms * 16;
    if (b > cap) b = cap;
    return int(b < 1 ? 1 : b);
}

}  // namespace

cudaError_t cavity3d_predict(const Cavity3dState &s, double dt, cudaStream_t st) {
    G3 g{s.nx, s.ny, s.nz, s.dx, s.dy, s.dz};
    predict_u<<<grid_for((long long)(s.nx + 1) * s.ny * s.nz, s.sms), kBlk, 0, st>>>(s.u, s.v, s.w, s.us, g, dt, s.nu, s.lid);
    predict_v<<<grid_for((long long)s.nx * (s.ny + 1) * s.nz, s.sms), kBlk, 0, st>>>(s.u, s.v, s.w, s.vs, g, dt, s.nu);
    predict_w<<<grid_for((long long)s.nx * s.ny * (s.nz + 1), s.sms), kBlk, 0, st>>>(s.u, s.v, s.w, s.ws, g, dt, s.nu);
    return cudaGetLastError();
}

cudaError_t cavity3d_rhs(const Cavity3dState &s, double dt, cudaStream_t st) {
    G3 g{s.nx, s.ny, s.nz, s.dx, s.dy, s.dz};
    build_rhs<<<grid_for((long long)s.nx * s.ny * s.nz, s.sms), kBlk, 0, st>>>(s.us, s.vs, s.ws, s.rhs, g, s.rho / dt);
    return cudaGetLastError();
}

cudaError_t cavity3d_correct(const Cavity3dState &s, double dt, cudaStream_t st) {
    G3 g{s.nx, s.ny, s.nz, s.dx, s.dy, s.dz};
    correct_all<<<grid_for((long long)s.nx * s.ny * s.nz, s.sms), kBlk, 0, st>>>(s.us, s.vs, s.ws, s.p, s.u, s.v, s.w,
                                                                                g, dt / s.rho);
    return cudaGetLastError();
}

cudaError_t cavity3d_diagnostics(const Cavity3dState &s, Diag3Dev *out, cudaStream_t st) {
    G3 g{s.nx, s.ny, s.nz, s.dx, s.dy, s.dz};
    diag_reset<<<1, 1, 0, st>>>(out);
    const long long n = (long long)(s.nx + 1) * (s.ny + 1) * (s.nz + 1);
    diagnostics<<<grid_for(n, s.sms), kBlk, 0, st>>>(s.u, s.v, s.w, s.p, g, out);
    return cudaGetLastError();
}

}  // namespace flursys
