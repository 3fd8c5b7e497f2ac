// cavity2d.cu — velocity phases of the 2D projection step
// (src/solver/incompressible.rs) on sm_100a, in FP64.
#include <cuda_runtime.h>

#include <cmath>

#include "cavity2d.cuh"
#include "common.cuh"
#include "pcg2d.cuh"

namespace flursys {

namespace {

constexpr int kBlk = 256;
constexpr int kPostParts = 8;

__device__ __forceinline__ bool sol(const Cavity2dState &s, int i, int j) {
    return (s.flags[i + s.nx * j] & kCellSolid) != 0;
}
// u_face_open / v_face_open (:2046-2064)
__device__ __forceinline__ bool u_open(const Cavity2dState &s, int i, int j) {
    if (i == 0) return !sol(s, 0, j);
    if (i == s.nx) return !sol(s, s.nx - 1, j);
    return !sol(s, i - 1, j) && !sol(s, i, j);
}
__device__ __forceinline__ bool v_open(const Cavity2dState &s, int i, int j) {
    if (j == 0) return !sol(s, i, 0);
    if (j == s.ny) return !sol(s, i, s.ny - 1);
    return !sol(s, i, j - 1) && !sol(s, i, j);
}

// MomentumStencil::u_neighbor (:2090-2122) with tangential_ghost_u (:2159-2178).
__device__ __forceinline__ double u_nb(const Cavity2dState &s, const double *u, int i, int j, int di, int dj,
                                       double c) {
    const int ii = i + di, jj = j + dj;
    if (ii >= 0 && ii <= s.nx && jj >= 0 && jj < s.ny) return u_open(s, ii, jj) ? u[ii + (s.nx + 1) * jj] : -c;
    if (jj < 0) return s.kind[2] == kBkVelocity ? 2.0 * s.gu_bottom[i] - c : c;
    if (jj >= s.ny) return s.kind[3] == kBkVelocity ? 2.0 * s.gu_top[i] - c : c;
    return c;
}
// MomentumStencil::v_neighbor (:2124-2156) with tangential_ghost_v (:2180-2199).
__device__ __forceinline__ double v_nb(const Cavity2dState &s, const double *v, int i, int j, int di, int dj,
                                       double c) {
    const int ii = i + di, jj = j + dj;
    if (ii >= 0 && ii < s.nx && jj >= 0 && jj <= s.ny) return v_open(s, ii, jj) ? v[ii + s.nx * jj] : -c;
    if (ii < 0) return s.kind[0] == kBkVelocity ? 2.0 * s.gv_left[j] - c : c;
    if (ii >= s.nx) return s.kind[1] == kBkVelocity ? 2.0 * s.gv_right[j] - c : c;
    return c;
}

// transported (:2201-2212)
__device__ __forceinline__ double transported(int scheme, double fv, double left, double right) {
    if (scheme == FLURSYS_CONVECTION_UPWIND) return fv >= 0.0 ? left : right;
    return 0.5 * (left + right);
}

// predict_momentum (:748-922) without buoyancy; every face is written.
__global__ void __launch_bounds__(kBlk) predict2d(Cavity2dState s, double dt, int with_p, double relax) {
    const int nu = (s.nx + 1) * s.ny, nv = s.nx * (s.ny + 1);
    const double *u = s.u, *v = s.v, *p = s.p;
    for (int id = blockIdx.x * kBlk + threadIdx.x; id < nu + nv; id += gridDim.x * kBlk) {
        if (id < nu) {
            const int j = id / (s.nx + 1), i = id - j * (s.nx + 1);
            if (i == 0 || i == s.nx || !u_open(s, i, j)) { s.us[id] = 0.0; continue; }
            const double up = u[id];
            const double ue_nb = u_nb(s, u, i, j, 1, 0, up), uw_nb = u_nb(s, u, i, j, -1, 0, up);
            const double un_nb = u_nb(s, u, i, j, 0, 1, up), us_nb = u_nb(s, u, i, j, 0, -1, up);
            const double ue = 0.5 * (up + ue_nb), uw = 0.5 * (uw_nb + up);
            const double vn = 0.5 * (v[i - 1 + s.nx * (j + 1)] + v[i + s.nx * (j + 1)]);
            const double vs = 0.5 * (v[i - 1 + s.nx * j] + v[i + s.nx * j]);
            const double pe = transported(s.convection, ue, up, ue_nb), pw = transported(s.convection, uw, uw_nb, up);
            const double pn = transported(s.convection, vn, up, un_nb), ps = transported(s.convection, vs, us_nb, up);
            const double conv = (ue * pe - uw * pw) / s.dx + (vn * pn - vs * ps) / s.dy;
            const double diff = (ue_nb - 2.0 * up + uw_nb) / (s.dx * s.dx) + (un_nb - 2.0 * up + us_nb) / (s.dy * s.dy);
            const double pg = with_p ? (p[i + s.nx * j] - p[i - 1 + s.nx * j]) / s.dx : 0.0;
            s.us[id] = up + relax * dt * (-conv + s.nu * diff - pg / s.rho);
        } else {
            const int vid = id - nu;
            const int j = vid / s.nx, i = vid - j * s.nx;
            if (j == 0 || j == s.ny || !v_open(s, i, j)) { s.vs[vid] = 0.0; continue; }
            const double vp = v[vid];
            const double ve_nb = v_nb(s, v, i, j, 1, 0, vp), vw_nb = v_nb(s, v, i, j, -1, 0, vp);
            const double vn_nb = v_nb(s, v, i, j, 0, 1, vp), vs_nb = v_nb(s, v, i, j, 0, -1, vp);
            const double ue = 0.5 * (u[i + 1 + (s.nx + 1) * (j - 1)] + u[i + 1 + (s.nx + 1) * j]);
            const double uw = 0.5 * (u[i + (s.nx + 1) * (j - 1)] + u[i + (s.nx + 1) * j]);
            const double vn = 0.5 * (vp + vn_nb), vs = 0.5 * (vs_nb + vp);
            const double pe = transported(s.convection, ue, vp, ve_nb), pw = transported(s.convection, uw, vw_nb, vp);
            const double pn = transported(s.convection, vn, vp, vn_nb), ps = transported(s.convection, vs, vs_nb, vp);
            const double conv = (ue * pe - uw * pw) / s.dx + (vn * pn - vs * ps) / s.dy;
            const double diff = (ve_nb - 2.0 * vp + vw_nb) / (s.dx * s.dx) + (vn_nb - 2.0 * vp + vs_nb) / (s.dy * s.dy);
            const double pg = with_p ? (p[i + s.nx * j] - p[i + s.nx * (j - 1)]) / s.dy : 0.0;
            s.vs[vid] = vp + relax * dt * (-conv + s.nu * diff - pg / s.rho);
        }
    }
}

// apply_velocity_boundaries (:1981-2027) on the normal boundary faces.
__global__ void boundaries2d(Cavity2dState s, double *u, double *v) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < s.ny) {
        const int j = t;
        const int su = s.nx + 1;
        switch (s.kind[0]) {
            case kBkVelocity: u[su * j] = s.bu_left[j]; break;
            case kBkSymmetry: u[su * j] = 0.0; break;
            default: u[su * j] = u[1 + su * j];
        }
        switch (s.kind[1]) {
            case kBkVelocity: u[s.nx + su * j] = s.bu_right[j]; break;
            case kBkSymmetry: u[s.nx + su * j] = 0.0; break;
            default: u[s.nx + su * j] = u[s.nx - 1 + su * j];
        }
    }
    if (t < s.nx) {
        const int i = t;
        switch (s.kind[2]) {
            case kBkVelocity: v[i] = s.bv_bottom[i]; break;
            case kBkSymmetry: v[i] = 0.0; break;
            default: v[i] = v[i + s.nx];
        }
        switch (s.kind[3]) {
            case kBkVelocity: v[i + s.nx * s.ny] = s.bv_top[i]; break;
            case kBkSymmetry: v[i + s.nx * s.ny] = 0.0; break;
            default: v[i + s.nx * s.ny] = v[i + s.nx * (s.ny - 1)];
        }
    }
}

// build_pressure_rhs (:924-970)
__global__ void __launch_bounds__(kBlk) rhs2d(Cavity2dState s, double rho_over_dt) {
    const int n = s.nx * s.ny;
    for (int c = blockIdx.x * kBlk + threadIdx.x; c < n; c += gridDim.x * kBlk) {
        if (s.flags[c] & 3) { s.rhs[c] = 0.0; continue; }
        const int j = c / s.nx, i = c - j * s.nx;
        const double div = (s.us[i + 1 + (s.nx + 1) * j] - s.us[i + (s.nx + 1) * j]) / s.dx +
                           (s.vs[i + s.nx * (j + 1)] - s.vs[i + s.nx * j]) / s.dy;
        s.rhs[c] = rho_over_dt * div;
    }
}

// correct_velocity (:1322-1379) into (un, vn).
__global__ void __launch_bounds__(kBlk) correct2d(Cavity2dState s, double dt_over_rho) {
    const int nu = (s.nx + 1) * s.ny, nv = s.nx * (s.ny + 1);
    for (int id = blockIdx.x * kBlk + threadIdx.x; id < nu + nv; id += gridDim.x * kBlk) {
        if (id < nu) {
            const int j = id / (s.nx + 1), i = id - j * (s.nx + 1);
            if (i == 0 || i == s.nx) { s.un[id] = s.us[id]; continue; }
            s.un[id] = u_open(s, i, j)
                           ? s.us[id] - dt_over_rho * ((s.p[i + s.nx * j] - s.p[i - 1 + s.nx * j]) / s.dx)
                           : 0.0;
        } else {
            const int vid = id - nu;
            const int j = vid / s.nx, i = vid - j * s.nx;
            if (j == 0 || j == s.ny) { s.vn[vid] = s.vs[vid]; continue; }
            s.vn[vid] = v_open(s, i, j)
                            ? s.vs[vid] - dt_over_rho * ((s.p[i + s.nx * j] - s.p[i + s.nx * (j - 1)]) / s.dy)
                            : 0.0;
        }
    }
}

// p = p_old + relax * p' (advance_one_step SIMPLE branch, :685-695)
__global__ void simple_relax2d(Cavity2dState s, double relax) {
    const int n = s.nx * s.ny;
    for (int c = blockIdx.x * kBlk + threadIdx.x; c < n; c += gridDim.x * kBlk) s.p[c] = s.pold[c] + relax * s.p[c];
}

__device__ __forceinline__ double vcell(const Cavity2dState &s, int i, int j) {
    return 0.5 * (s.vn[i + s.nx * j] + s.vn[i + s.nx * (j + 1)]);
}
__device__ __forceinline__ double ucell(const Cavity2dState &s, int i, int j) {
    return 0.5 * (s.un[i + (s.nx + 1) * j] + s.un[i + 1 + (s.nx + 1) * j]);
}

__global__ void __launch_bounds__(kBlk) post2d(Cavity2dState s) {
    __shared__ double red[kBlk / 32];
    const int nc = s.nx * s.ny, nu = (s.nx + 1) * s.ny, nv = s.nx * (s.ny + 1);
    const int nmax = max(nc, max(nu, nv));
    double mdiv = 0.0, mspeed = 0.0, mu = 0.0, mv = 0.0, du = 0.0, dv = 0.0, fx = 0.0, fy = 0.0;
    for (int id = blockIdx.x * kBlk + threadIdx.x; id < nmax; id += gridDim.x * kBlk) {
        if (id < nc) {
            const int j = id / s.nx, i = id - j * s.nx;
            if (sol(s, i, j)) {
                s.uc[id] = 0.0; s.vc[id] = 0.0; s.speed[id] = 0.0; s.vort[id] = 0.0;
            } else {
                const double a = ucell(s, i, j), b = vcell(s, i, j);
                const double sp = sqrt(a * a + b * b);
                s.uc[id] = a; s.vc[id] = b; s.speed[id] = sp;
                mspeed = fmax(mspeed, sp);
                if (!isfinite(sp)) atomicMin(&s.diag->bad_index[3], (unsigned long long)id);
                // derivative_x_slice / derivative_y_slice (:2227-2285)
                const bool e_ok = i + 1 < s.nx && !sol(s, i + 1, j), w_ok = i > 0 && !sol(s, i - 1, j);
                const bool n_ok = j + 1 < s.ny && !sol(s, i, j + 1), s_ok = j > 0 && !sol(s, i, j - 1);
                double dvdx = 0.0, dudy = 0.0;
                if (e_ok && w_ok) dvdx = (vcell(s, i + 1, j) - vcell(s, i - 1, j)) / (2.0 * s.dx);
                else if (e_ok) dvdx = (vcell(s, i + 1, j) - b) / s.dx;
                else if (w_ok) dvdx = (b - vcell(s, i - 1, j)) / s.dx;
                if (n_ok && s_ok) dudy = (ucell(s, i, j + 1) - ucell(s, i, j - 1)) / (2.0 * s.dy);
                else if (n_ok) dudy = (ucell(s, i, j + 1) - a) / s.dy;
                else if (s_ok) dudy = (a - ucell(s, i, j - 1)) / s.dy;
                s.vort[id] = dvdx - dudy;
                const double div = (s.un[i + 1 + (s.nx + 1) * j] - s.un[i + (s.nx + 1) * j]) / s.dx +
                                   (s.vn[i + s.nx * (j + 1)] - s.vn[i + s.nx * j]) / s.dy;
                mdiv = fmax(mdiv, fabs(div));
                if (s.cylinder) {  // cylinder_force_coefficients (:1642-1668)
                    const double pp = s.p[id];
                    if (i + 1 < s.nx && sol(s, i + 1, j)) { fx += pp * s.dy; fy += s.cylinder_mu * b / (0.5 * s.dx) * s.dy; }
                    if (i > 0 && sol(s, i - 1, j)) { fx -= pp * s.dy; fy += s.cylinder_mu * b / (0.5 * s.dx) * s.dy; }
                    if (j + 1 < s.ny && sol(s, i, j + 1)) { fy += pp * s.dx; fx += s.cylinder_mu * a / (0.5 * s.dy) * s.dx; }
                    if (j > 0 && sol(s, i, j - 1)) { fy -= pp * s.dx; fx += s.cylinder_mu * a / (0.5 * s.dy) * s.dx; }
                }
            }
            if (!isfinite(s.p[id])) atomicMin(&s.diag->bad_index[0], (unsigned long long)id);
        }
        if (id < nu) {
            const double a = s.un[id];
            mu = fmax(mu, fabs(a));
            du = fmax(du, fabs(a - s.u[id]));
            if (!isfinite(a)) atomicMin(&s.diag->bad_index[1], (unsigned long long)id);
        }
        if (id < nv) {
            const double b = s.vn[id];
            mv = fmax(mv, fabs(b));
            dv = fmax(dv, fabs(b - s.v[id]));
            if (!isfinite(b)) atomicMin(&s.diag->bad_index[2], (unsigned long long)id);
        }
    }
    const double vals[kPostParts] = {mdiv, mspeed, mu, mv, du, dv, fx, fy};
    for (int k = 0; k < kPostParts; ++k) {
        const double t = k < 6 ? block_max<kBlk>(vals[k], red) : block_sum<kBlk>(vals[k], red);
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
            a = k < 6 ? fmax(a, v) : a + v;
        }
        out[k] = k < 6 ? block_max<kBlk>(a, red) : block_sum<kBlk>(a, red);
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
    }
}

__global__ void diag2d_reset(Diag2Dev *d) {
    for (int f = 0; f < 4; ++f) d->bad_index[f] = ~0ull;
}

int grid_for(long long n, int sms) {
    long long b = (n + kBlk - 1) / kBlk;
    const long long cap = (long long)sms * 8;
    if (b > cap) b = cap;
    return int(b < 1 ? 1 : b);
}

}  // namespace

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

cudaError_t cavity2d_post(const Cavity2dState &s, cudaStream_t st) {
    diag2d_reset<<<1, 1, 0, st>>>(s.diag);
    post2d<<<s.post_blocks, kBlk, 0, st>>>(s);
    post2d_finalize<<<1, kBlk, 0, st>>>(s);
    return cudaGetLastError();
}

}  // namespace flursys
