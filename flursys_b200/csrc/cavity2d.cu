// cavity2d.cu — velocity phases of the 2D projection step
// (src/solver/incompressible.rs) on sm_100a, in FP64; the per-element work
// lives in cavity2d_dev.cuh.
#include <cuda_runtime.h>

#include <cmath>

#include "cavity2d.cuh"
#include "cavity2d_dev.cuh"
#include "common.cuh"
#include "pcg2d.cuh"

namespace flursys {

namespace {

constexpr int kBlk = 256;
constexpr int kPostParts = 10;

__global__ void __launch_bounds__(kBlk) predict2d(Cavity2dState s, double dt, int with_p, double relax) {
    const int n = (s.nx + 1) * s.ny + s.nx * (s.ny + 1);
    for (int id = blockIdx.x * kBlk + threadIdx.x; id < n; id += gridDim.x * kBlk) predict_elem(s, id, dt, with_p, relax);
}

__global__ void boundaries2d(Cavity2dState s, double *u, double *v) {
    boundary_elem(s, u, v, blockIdx.x * blockDim.x + threadIdx.x);
}

__global__ void __launch_bounds__(kBlk) rhs2d(Cavity2dState s, double rho_over_dt) {
    const int n = s.nx * s.ny;
    for (int c = blockIdx.x * kBlk + threadIdx.x; c < n; c += gridDim.x * kBlk) rhs_elem(s, c, rho_over_dt);
}

__global__ void __launch_bounds__(kBlk) correct2d(Cavity2dState s, double dt_over_rho) {
    const int n = (s.nx + 1) * s.ny + s.nx * (s.ny + 1);
    for (int id = blockIdx.x * kBlk + threadIdx.x; id < n; id += gridDim.x * kBlk) correct_elem(s, id, dt_over_rho);
}

// p = p_old + relax * p' (advance_one_step SIMPLE branch, :685-695)
__global__ void simple_relax2d(Cavity2dState s, double relax) {
    const int n = s.nx * s.ny;
    for (int c = blockIdx.x * kBlk + threadIdx.x; c < n; c += gridDim.x * kBlk) s.p[c] = s.pold[c] + relax * s.p[c];
}

// Parts 6 and 7 (force sums) add up; every other part is a maximum.
__device__ __forceinline__ bool is_max_part(int k) { return k != 6 && k != 7; }

__global__ void __launch_bounds__(kBlk) post2d(Cavity2dState s) {
    __shared__ double red[kBlk / 32];
    const int nc = s.nx * s.ny, nu = (s.nx + 1) * s.ny, nv = s.nx * (s.ny + 1);
    const int nmax = max(nc, max(nu, nv));
    PostAcc a;
    for (int id = blockIdx.x * kBlk + threadIdx.x; id < nmax; id += gridDim.x * kBlk) post_elem(s, id, a);
    const double vals[kPostParts] = {a.mdiv, a.mspeed, a.mu, a.mv, a.du, a.dv, a.fx, a.fy, a.muc, a.mvc};
    for (int k = 0; k < kPostParts; ++k) {
        const double t = is_max_part(k) ? block_max<kBlk>(vals[k], red) : block_sum<kBlk>(vals[k], red);
        if (threadIdx.x == 0) s.partials[blockIdx.x * kPostParts + k] = t;
    }
}

// Fixed-order final reduction of the post-pass partials.
__global__ void post2d_finalize(Cavity2dState s) {
    __shared__ double red[kBlk / 32];
    double out[kPostParts];
    for (int k = 0; k < kPostParts; ++k) {
        double a = 0.0;
        for (int b = threadIdx.x; b < s.post_blocks; b += kBlk) {
            const double v = s.partials[b * kPostParts + k];
            a = is_max_part(k) ? fmax(a, v) : a + v;
        }
        out[k] = is_max_part(k) ? block_max<kBlk>(a, red) : block_sum<kBlk>(a, red);
    }
    if (threadIdx.x == 0) {
        Diag2Dev *d = s.diag;
        d->max_divergence = out[0];
        d->max_speed = out[1];
        d->max_abs_u = out[2];
        d->max_abs_v = out[3];
        d->du = out[4];
        d->dv = out[5];
        d->fx = out[6];
        d->fy = out[7];
        d->max_abs_uc = out[8];
        d->max_abs_vc = out[9];
    }
}

__global__ void diag2d_reset(Diag2Dev *d) {
    for (int f = 0; f < 5; ++f) d->bad_index[f] = ~0ull;
}

__global__ void __launch_bounds__(kBlk) temperature2d(Cavity2dState s, double dt) {
    const int n = s.nx * s.ny;
    for (int c = blockIdx.x * kBlk + threadIdx.x; c < n; c += gridDim.x * kBlk) temperature_elem(s, c, dt);
}

int grid_for(long long n, int sms) {
    long long b = (n + kBlk - 1) / kBlk;
    const long long cap = (long long)sms * 8;
    if (b > cap) b = cap;
    return int(b < 1 ? 1 : b);
}

}  // namespace

int cavity2d_post_parts() { return kPostParts; }

int cavity2d_post_blocks(int nx, int ny, int sms) {
    return grid_for((long long)(nx + 1) * (ny + 1), sms);
}

cudaError_t cavity2d_predict(const Cavity2dState &s, double dt, int with_pressure, double relax, cudaStream_t st) {
    predict2d<<<grid_for((long long)(s.nx + 1) * s.ny + (long long)s.nx * (s.ny + 1), s.sms), kBlk, 0, st>>>(
        s, dt, with_pressure, relax);
    return cudaGetLastError();
}

cudaError_t cavity2d_boundaries(const Cavity2dState &s, double *u, double *v, cudaStream_t st) {
    const int n = s.nx > s.ny ? s.nx : s.ny;
    boundaries2d<<<(n + 127) / 128, 128, 0, st>>>(s, u, v);
    return cudaGetLastError();
}

cudaError_t cavity2d_rhs(const Cavity2dState &s, double rho_over_dt, cudaStream_t st) {
    rhs2d<<<grid_for((long long)s.nx * s.ny, s.sms), kBlk, 0, st>>>(s, rho_over_dt);
    return cudaGetLastError();
}

cudaError_t cavity2d_correct(const Cavity2dState &s, double dt_over_rho, cudaStream_t st) {
    correct2d<<<grid_for((long long)(s.nx + 1) * s.ny + (long long)s.nx * (s.ny + 1), s.sms), kBlk, 0, st>>>(
        s, dt_over_rho);
    return cudaGetLastError();
}

cudaError_t cavity2d_simple_relax(const Cavity2dState &s, double relax, cudaStream_t st) {
    simple_relax2d<<<grid_for((long long)s.nx * s.ny, s.sms), kBlk, 0, st>>>(s, relax);
    return cudaGetLastError();
}

cudaError_t cavity2d_temperature(const Cavity2dState &s, double dt, cudaStream_t st) {
    temperature2d<<<grid_for((long long)s.nx * s.ny, s.sms), kBlk, 0, st>>>(s, dt);
    return cudaGetLastError();
}

cudaError_t cavity2d_post(const Cavity2dState &s, cudaStream_t st) {
    diag2d_reset<<<1, 1, 0, st>>>(s.diag);
    post2d<<<s.post_blocks, kBlk, 0, st>>>(s);
    post2d_finalize<<<1, kBlk, 0, st>>>(s);
    return cudaGetLastError();
}

}  // namespace flursys
