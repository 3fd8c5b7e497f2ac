// simple2d.cu — steady collocated SIMPLE on the plane channel
// (flursys_cuda_simple_channel): solve_incompressible
// (src/unstructured_incompressible.rs:368-482) with solve_simple
// (src/simple.rs:148-314) on nx x ny uniform quads of unit depth.
//
// The reference's face-based operators are evaluated in cell/face index
// space: cell c = i + nx j; x-faces f = i + (nx + 1) j (i = 0 the inlet,
// i = nx the outlet), y-faces g = i + nx j (j = 0 and j = ny the walls).
// Face fluxes are stored positive along +x / +y; the reference's
// owner-oriented flux of a boundary face is -F on the inlet and the bottom
// wall and +F on the outlet and the top wall. Every per-face quantity keeps
// the reference's arithmetic (interpolation weight (x_f - x_P).d / d.d,
// (S.d)/(d.d) coefficients, sums in the reference's face order), so the
// device and the FP64 oracle differ only by the Krylov solves' reduction
// order.
//
// One outer iteration, all on the device (one host synchronisation at its
// end to read the linear-solve reports and the continuity RMS):
//   k_grad          least-squares pressure gradient (numerics.rs:106-200,650-682)
//   k_momentum      5-point momentum CSR + both right-hand sides + rAU
//                   (momentum.rs:180-341; the x and y systems share their
//                   matrix: same flux, viscosity and boundary kinds)
//   BiCGSTAB x2     csr.cu, device-resident (the z system is identically zero
//                   on a 2D mesh: the reference solves it in 0 iterations)
//   k_rhie_chow     predicted face flux and d_f (simple.rs:342-410,757-805)
//   k_passemble     pressure-correction CSR with the fixed outlet
//                   (simple.rs:583-643)
//   Jacobi-PCG      csr.cu
//   k_grad, k_velocity, k_flux   p += a_p p', U = U* - rAU grad p',
//                   Phi = Phi* - d_f (p'_N - p'_P) (simple.rs:448-496,673-704)
//   k_continuity    integrated divergence, RMS (simple.rs:706-718)
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "capi_internal.cuh"
#include "common.cuh"
#include "csr.cuh"
#include "flursys_cuda.h"

namespace flursys {

namespace {

constexpr int kBlk = 256;

struct Chan {
    int nx, ny;
    double L, H, dx, dy, nu, alpha_u, peak, pout;
    const int *ro;  // 5-point CSR row offsets (columns S, W, P, E, N where present)
};

__device__ __forceinline__ double cxp(const Chan &g, int i) { return (i + 0.5) * g.dx; }
__device__ __forceinline__ double cyp(const Chan &g, int j) { return (j + 0.5) * g.dy; }

// Least-squares gradient of a cell field with the pressure boundary
// conditions: zero gradient on the inlet and the walls (no equation),
// fixed value `fixed` on the outlet. Equations in the cell's face order
// W, E, S, N, outlet.
__global__ void __launch_bounds__(kBlk) k_grad(Chan g, const double *__restrict__ phi, double fixed, double *gx,
                                               double *gy) {
    const int n = g.nx * g.ny;
    for (int c = blockIdx.x * kBlk + threadIdx.x; c < n; c += gridDim.x * kBlk) {
        const int j = c / g.nx, i = c - j * g.nx;
        const double pc = phi[c];
        double n0 = 0.0, n4 = 0.0, rx = 0.0, ry = 0.0;
        auto eqx = [&](double off, double adj) {
            const double w = 1.0 / (off * off);
            const double rc = off * w;
            n0 += rc * off;
            rx += rc * (adj - pc);
        };
        auto eqy = [&](double off, double adj) {
            const double w = 1.0 / (off * off);
            const double rc = off * w;
            n4 += rc * off;
            ry += rc * (adj - pc);
        };
        if (i > 0) eqx(cxp(g, i - 1) - cxp(g, i), phi[c - 1]);
        if (i + 1 < g.nx) eqx(cxp(g, i + 1) - cxp(g, i), phi[c + 1]);
        if (j > 0) eqy(cyp(g, j - 1) - cyp(g, j), phi[c - g.nx]);
        if (j + 1 < g.ny) eqy(cyp(g, j + 1) - cyp(g, j), phi[c + g.nx]);
        if (i + 1 == g.nx) eqx(g.L - cxp(g, i), fixed);
        const double det = n0 * n4 - 0.0 * 0.0;
        gx[c] = (n4 / det) * rx + (-0.0 / det) * ry;
        gy[c] = (-0.0 / det) * rx + (n0 / det) * ry;
    }
}

// Momentum system of one outer iteration (both components).
__global__ void __launch_bounds__(kBlk) k_momentum(Chan g, const double *__restrict__ Fx, const double *__restrict__ Fy,
                                                   const double *__restrict__ gx, const double *__restrict__ gy,
                                                   const double *__restrict__ u, const double *__restrict__ v,
                                                   double *vals, double *bu, double *bv, double *rau, int *flag) {
    const int n = g.nx * g.ny;
    const double vol = g.dx * g.dy;
    for (int c = blockIdx.x * kBlk + threadIdx.x; c < n; c += gridDim.x * kBlk) {
        const int j = c / g.nx, i = c - j * g.nx;
        double dg = 0.0, aS = 0.0, aW = 0.0, aE = 0.0, aN = 0.0;
        double ru = -gx[c] * vol, rv = -gy[c] * vol;
        // internal faces in face order: x-faces (W: this cell is the
        // neighbour, E: the owner), then y-faces (S, N)
        if (i > 0) {
            const double d = cxp(g, i) - cxp(g, i - 1), D = g.nu * (g.dy * d) / (d * d), phi = Fx[i + (g.nx + 1) * j];
            aW = -D - fmax(phi, 0.0);
            dg += D - fmin(phi, 0.0);
        }
        if (i + 1 < g.nx) {
            const double d = cxp(g, i + 1) - cxp(g, i), D = g.nu * (g.dy * d) / (d * d), phi = Fx[i + 1 + (g.nx + 1) * j];
            dg += D + fmax(phi, 0.0);
            aE = -D + fmin(phi, 0.0);
        }
        if (j > 0) {
            const double d = cyp(g, j) - cyp(g, j - 1), D = g.nu * (g.dx * d) / (d * d), phi = Fy[i + g.nx * j];
            aS = -D - fmax(phi, 0.0);
            dg += D - fmin(phi, 0.0);
        }
        if (j + 1 < g.ny) {
            const double d = cyp(g, j + 1) - cyp(g, j), D = g.nu * (g.dx * d) / (d * d), phi = Fy[i + g.nx * (j + 1)];
            dg += D + fmax(phi, 0.0);
            aN = -D + fmin(phi, 0.0);
        }
        // boundary faces in patch order: inlet, outlet, bottom, top
        auto fixed_face = [&](double sd, double dd, double phi, double val_u, double val_v) {
            const double D = g.nu * sd / dd;
            dg += D + fmax(phi, 0.0);
            ru += D * val_u - fmin(phi, 0.0) * val_u;
            rv += D * val_v - fmin(phi, 0.0) * val_v;
        };
        if (i == 0) {
            const double d = 0.0 - cxp(g, 0), y = cyp(g, j);
            const double uin = g.peak * 4.0 * y * (g.H - y) / (g.H * g.H);
            fixed_face((-g.dy) * d, d * d, -Fx[(g.nx + 1) * j], uin, 0.0);
        }
        if (i + 1 == g.nx) {  // zero gradient
            const double phi = Fx[g.nx + (g.nx + 1) * j];
            if (phi < 0.0) atomicOr(flag, 1);
            dg += phi;
        }
        if (j == 0) {
            const double d = 0.0 - cyp(g, 0);
            fixed_face((-g.dx) * d, d * d, -Fy[i], 0.0, 0.0);
        }
        if (j + 1 == g.ny) {
            const double d = g.H - cyp(g, j);
            fixed_face(g.dx * d, d * d, Fy[i + g.nx * g.ny], 0.0, 0.0);
        }
        // equation under-relaxation (momentum.rs:301-333)
        const double a = g.alpha_u;
        double dr = dg;
        if (a != 1.0) {
            dr = dg / a;
            ru += (1.0 - a) / a * dg * u[c];
            rv += (1.0 - a) / a * dg * v[c];
        }
        double *row = vals + g.ro[c];
        int k = 0;
        if (j > 0) row[k++] = aS;
        if (i > 0) row[k++] = aW;
        row[k++] = dr;
        if (i + 1 < g.nx) row[k++] = aE;
        if (j + 1 < g.ny) row[k++] = aN;
        bu[c] = ru;
        bv[c] = rv;
        if (!(isfinite(dr) && dr > 0.0)) atomicOr(flag, 2);
        rau[c] = 1.0 / dr;
    }
}

// Rhie-Chow predicted flux and the pressure-response coefficients.
__global__ void __launch_bounds__(kBlk) k_rhie_chow(Chan g, const double *__restrict__ us, const double *__restrict__ vs,
                                                    const double *__restrict__ p, const double *__restrict__ gx,
                                                    const double *__restrict__ gy, const double *__restrict__ rau,
                                                    const double *__restrict__ Fx, const double *__restrict__ Fy,
                                                    double *Fxp, double *Fyp, double *cfx, double *cfy) {
    const int nfx = (g.nx + 1) * g.ny, nfy = g.nx * (g.ny + 1);
    for (int t = blockIdx.x * kBlk + threadIdx.x; t < nfx + nfy; t += gridDim.x * kBlk) {
        if (t < nfx) {
            const int j = t / (g.nx + 1), i = t - j * (g.nx + 1);
            if (i == 0) {  // inlet: prescribed flux
                Fxp[t] = Fx[t];
                cfx[t] = 0.0;
            } else if (i == g.nx) {  // outlet: predictor flux, fixed-correction coefficient
                const int o = g.nx - 1 + g.nx * j;
                const double d = g.L - cxp(g, g.nx - 1);
                Fxp[t] = us[o] * g.dy;
                cfx[t] = rau[o] * (g.dy * d) / (d * d);
            } else {
                const int o = i - 1 + g.nx * j, nb = o + 1;
                const double d = cxp(g, i) - cxp(g, i - 1);
                const double l = ((i * g.dx) - cxp(g, i - 1)) * d / (d * d);
                const double coef = (rau[o] * (1.0 - l) + rau[nb] * l) * (g.dy * d) / (d * d);
                const double fu = us[o] * (1.0 - l) + us[nb] * l;
                const double fr = gx[o] * rau[o] * (1.0 - l) + gx[nb] * rau[nb] * l;
                Fxp[t] = fu * g.dy + fr * g.dy - coef * (p[nb] - p[o]);
                cfx[t] = coef;
            }
        } else {
            const int f = t - nfx;
            const int j = f / g.nx, i = f - j * g.nx;
            if (j == 0 || j == g.ny) {  // walls: prescribed flux
                Fyp[f] = Fy[f];
                cfy[f] = 0.0;
            } else {
                const int o = i + g.nx * (j - 1), nb = o + g.nx;
                const double d = cyp(g, j) - cyp(g, j - 1);
                const double l = ((j * g.dy) - cyp(g, j - 1)) * d / (d * d);
                const double coef = (rau[o] * (1.0 - l) + rau[nb] * l) * (g.dx * d) / (d * d);
                const double fv = vs[o] * (1.0 - l) + vs[nb] * l;
                const double fr = gy[o] * rau[o] * (1.0 - l) + gy[nb] * rau[nb] * l;
                Fyp[f] = fv * g.dx + fr * g.dx - coef * (p[nb] - p[o]);
                cfy[f] = coef;
            }
        }
    }
}

// Pressure-correction system: -div(Phi*) with the fixed outlet correction 0.
__global__ void __launch_bounds__(kBlk) k_passemble(Chan g, const double *__restrict__ Fxp,
                                                    const double *__restrict__ Fyp, const double *__restrict__ cfx,
                                                    const double *__restrict__ cfy, double *vals, double *rhs) {
    const int n = g.nx * g.ny;
    for (int c = blockIdx.x * kBlk + threadIdx.x; c < n; c += gridDim.x * kBlk) {
        const int j = c / g.nx, i = c - j * g.nx;
        const int fw = i + (g.nx + 1) * j, fs = i + g.nx * j;
        double r = 0.0, dg = 0.0, aS = 0.0, aW = 0.0, aE = 0.0, aN = 0.0;
        if (i > 0) { r += Fxp[fw]; dg += cfx[fw]; aW = -cfx[fw]; }
        if (i + 1 < g.nx) { r -= Fxp[fw + 1]; dg += cfx[fw + 1]; aE = -cfx[fw + 1]; }
        if (j > 0) { r += Fyp[fs]; dg += cfy[fs]; aS = -cfy[fs]; }
        if (j + 1 < g.ny) { r -= Fyp[fs + g.nx]; dg += cfy[fs + g.nx]; aN = -cfy[fs + g.nx]; }
        if (i == 0) r -= -Fxp[fw];
        if (i + 1 == g.nx) {
            r -= Fxp[fw + 1];
            dg += cfx[fw + 1];
            r += cfx[fw + 1] * 0.0;
        }
        if (j == 0) r -= -Fyp[fs];
        if (j + 1 == g.ny) r -= Fyp[fs + g.nx];
        double *row = vals + g.ro[c];
        int k = 0;
        if (j > 0) row[k++] = aS;
        if (i > 0) row[k++] = aW;
        row[k++] = dg;
        if (i + 1 < g.nx) row[k++] = aE;
        if (j + 1 < g.ny) row[k++] = aN;
        rhs[c] = r;
    }
}

// p += a_p p'; U = U* - rAU grad p'.
__global__ void __launch_bounds__(kBlk) k_velocity(int n, double ap, const double *__restrict__ pc, double *p,
                                                   const double *__restrict__ us, const double *__restrict__ vs,
                                                   const double *__restrict__ rau, const double *__restrict__ gx,
                                                   const double *__restrict__ gy, double *u, double *v) {
    for (int c = blockIdx.x * kBlk + threadIdx.x; c < n; c += gridDim.x * kBlk) {
        p[c] += ap * pc[c];
        u[c] = us[c] - gx[c] * rau[c];
        v[c] = vs[c] - gy[c] * rau[c];
    }
}

// Phi = Phi* - d_f (p'_N - p'_P) on internal and fixed-correction faces.
__global__ void __launch_bounds__(kBlk) k_flux(Chan g, const double *__restrict__ Fxp, const double *__restrict__ Fyp,
                                               const double *__restrict__ cfx, const double *__restrict__ cfy,
                                               const double *__restrict__ pc, double *Fx, double *Fy) {
    const int nfx = (g.nx + 1) * g.ny, nfy = g.nx * (g.ny + 1);
    for (int t = blockIdx.x * kBlk + threadIdx.x; t < nfx + nfy; t += gridDim.x * kBlk) {
        if (t < nfx) {
            const int j = t / (g.nx + 1), i = t - j * (g.nx + 1);
            double f = Fxp[t];
            if (i == g.nx) f -= cfx[t] * (0.0 - pc[g.nx - 1 + g.nx * j]);
            else if (i > 0) f -= cfx[t] * (pc[i + g.nx * j] - pc[i - 1 + g.nx * j]);
            Fx[t] = f;
        } else {
            const int e = t - nfx;
            const int j = e / g.nx, i = e - j * g.nx;
            double f = Fyp[e];
            if (j > 0 && j < g.ny) f -= cfy[e] * (pc[i + g.nx * j] - pc[i + g.nx * (j - 1)]);
            Fy[e] = f;
        }
    }
}

// Per-block partial sums of the squared integrated divergence.
__global__ void __launch_bounds__(kBlk) k_continuity(Chan g, const double *__restrict__ Fx,
                                                     const double *__restrict__ Fy, double *partials) {
    __shared__ double red[kBlk / 32];
    const int n = g.nx * g.ny;
    double s = 0.0;
    for (int c = blockIdx.x * kBlk + threadIdx.x; c < n; c += gridDim.x * kBlk) {
        const int j = c / g.nx, i = c - j * g.nx;
        const int fw = i + (g.nx + 1) * j, fs = i + g.nx * j;
        double d = 0.0;  // internal faces first, then boundary faces (face order)
        if (i > 0) d -= Fx[fw];
        if (i + 1 < g.nx) d += Fx[fw + 1];
        if (j > 0) d -= Fy[fs];
        if (j + 1 < g.ny) d += Fy[fs + g.nx];
        if (i == 0) d += -Fx[fw];
        if (i + 1 == g.nx) d += Fx[fw + 1];
        if (j == 0) d += -Fy[fs];
        if (j + 1 == g.ny) d += Fy[fs + g.nx];
        s += d * d;
    }
    s = block_sum<kBlk>(s, red);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

int grid_for(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + kBlk - 1) / kBlk, 148 * 8)); }

int32_t fail(std::string *err, const std::string &msg, int32_t code) {
    *err = msg;
    return code;
}

}  // namespace

int32_t simple_channel_device(const FlursysSimpleConfig &c, double *hu, double *hv, double *hp, double *hflux,
                              double *hhist, FlursysSimpleReport *rep, std::string *err) {
    std::memset(rep, 0, sizeof *rep);
    if (c.abi_version != FLURSYS_CUDA_ABI_VERSION) return fail(err, "config abi_version does not match the library", FLURSYS_ERR_INVALID_ARGUMENT);
    if (c.nx < 2 || c.ny < 2 || (c.nx + 1) * (c.ny + 1) * 5 >= (1LL << 31))
        return fail(err, "nx and ny must be at least 2 and the matrix below 2^31 entries", FLURSYS_ERR_INVALID_CONFIG);
    if (!(c.length > 0.0 && c.height > 0.0 && std::isfinite(c.length) && std::isfinite(c.height)))
        return fail(err, "Domain dimensions must be positive", FLURSYS_ERR_INVALID_CONFIG);
    if (!(std::isfinite(c.kinematic_viscosity) && c.kinematic_viscosity >= 0.0))
        return fail(err, "kinematic viscosity must be finite and non-negative", FLURSYS_ERR_INVALID_CONFIG);
    if (!std::isfinite(c.inlet_peak_velocity) || !std::isfinite(c.outlet_pressure))
        return fail(err, "inlet velocity and outlet pressure must be finite", FLURSYS_ERR_INVALID_CONFIG);
    if (c.max_outer_iterations < 1) return fail(err, "max_outer_iterations must be positive", FLURSYS_ERR_INVALID_CONFIG);
    if (!(c.pressure_relaxation > 0.0 && c.pressure_relaxation <= 1.0))
        return fail(err, "pressure relaxation must lie in (0, 1]", FLURSYS_ERR_INVALID_CONFIG);
    if (!(c.velocity_relaxation > 0.0 && c.velocity_relaxation <= 1.0))
        return fail(err, "momentum under-relaxation must lie in (0, 1]", FLURSYS_ERR_INVALID_CONFIG);
    if (!(std::isfinite(c.continuity_tolerance) && c.continuity_tolerance >= 0.0))
        return fail(err, "continuity tolerance must be finite and non-negative", FLURSYS_ERR_INVALID_CONFIG);
    const int nx = (int)c.nx, ny = (int)c.ny, n = nx * ny;
    const int nfx = (nx + 1) * ny, nfy = nx * (ny + 1);
    // 5-point pattern
    std::vector<int> ro(n + 1), ci;
    ci.reserve((size_t)n * 5);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const int cc = i + nx * j;
            ro[cc] = (int)ci.size();
            if (j > 0) ci.push_back(cc - nx);
            if (i > 0) ci.push_back(cc - 1);
            ci.push_back(cc);
            if (i + 1 < nx) ci.push_back(cc + 1);
            if (j + 1 < ny) ci.push_back(cc + nx);
        }
    ro[n] = (int)ci.size();
    const int nnz = ro[n];
    int device = 0;
    cudaGetDevice(&device);
    cudaStream_t st;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return set_cuda_error(err, e, "SIMPLE stream");
    std::vector<void *> allocs;
    auto dalloc = [&](size_t bytes) -> void * {
        void *q = nullptr;
        if (e == cudaSuccess) e = cudaMalloc(&q, std::max<size_t>(bytes, 8));
        if (e == cudaSuccess) {
            allocs.push_back(q);
            e = cudaMemsetAsync(q, 0, std::max<size_t>(bytes, 8), st);
        }
        return q;
    };
    int *d_ro = (int *)dalloc(sizeof(int) * (n + 1));
    int *d_ci = (int *)dalloc(sizeof(int) * nnz);
    double *mvals = (double *)dalloc(8.0 * nnz), *pvals = (double *)dalloc(8.0 * nnz);
    double *u = (double *)dalloc(8.0 * n), *v = (double *)dalloc(8.0 * n), *p = (double *)dalloc(8.0 * n);
    double *us = (double *)dalloc(8.0 * n), *vs = (double *)dalloc(8.0 * n), *pc = (double *)dalloc(8.0 * n);
    double *gx = (double *)dalloc(8.0 * n), *gy = (double *)dalloc(8.0 * n), *rau = (double *)dalloc(8.0 * n);
    double *bu = (double *)dalloc(8.0 * n), *bv = (double *)dalloc(8.0 * n), *prhs = (double *)dalloc(8.0 * n);
    double *Fx = (double *)dalloc(8.0 * nfx), *Fy = (double *)dalloc(8.0 * nfy);
    double *Fxp = (double *)dalloc(8.0 * nfx), *Fyp = (double *)dalloc(8.0 * nfy);
    double *cfx = (double *)dalloc(8.0 * nfx), *cfy = (double *)dalloc(8.0 * nfy);
    const int ncb = grid_for(n);
    double *part = (double *)dalloc(8.0 * ncb);
    int *flag = (int *)dalloc(sizeof(int));
    double *h_part = nullptr;
    int *h_flag = nullptr;
    if (e == cudaSuccess) e = cudaMallocHost(&h_part, 8 * ncb);
    if (e == cudaSuccess) e = cudaMallocHost(&h_flag, sizeof(int));
    CsrDeviceWork wu, wv, wp;
    if (e == cudaSuccess) e = wu.ensure(n, device);
    if (e == cudaSuccess) e = wv.ensure(n, device);
    if (e == cudaSuccess) e = wp.ensure(n, device);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_ro, ro.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_ci, ci.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice, st);
    // initial_face_flux: zero initial velocity; the inlet's prescribed flux
    // (owner-oriented u_in * (-dy), i.e. +x flux u_in * dy); walls 0.
    std::vector<double> fx0(nfx, 0.0);
    const double dx = c.length / nx, dy = c.height / ny;
    for (int j = 0; j < ny; ++j) {
        const double y = (j + 0.5) * dy;
        const double uin = c.inlet_peak_velocity * 4.0 * y * (c.height - y) / (c.height * c.height);
        fx0[(nx + 1) * j] = -(uin * (-dy));
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(Fx, fx0.data(), 8 * nfx, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    int32_t status = FLURSYS_OK;
    std::vector<double> hist;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e != cudaSuccess) status = set_cuda_error(err, e, "SIMPLE set-up");
    Chan g{nx, ny, c.length, c.height, dx, dy, c.kinematic_viscosity, c.velocity_relaxation, c.inlet_peak_velocity,
           c.outlet_pressure, d_ro};
    auto continuity = [&](double *out) -> cudaError_t {
        k_continuity<<<ncb, kBlk, 0, st>>>(g, Fx, Fy, part);
        cudaError_t m = cudaMemcpyAsync(h_part, part, 8 * ncb, cudaMemcpyDeviceToHost, st);
        if (m == cudaSuccess) m = cudaStreamSynchronize(st);
        double s = 0.0;
        for (int b = 0; b < ncb; ++b) s += h_part[b];
        *out = std::sqrt(s / double(n));
        return m;
    };
    if (!status) {
        double c0 = 0.0;
        e = continuity(&c0);
        if (e != cudaSuccess) status = set_cuda_error(err, e, "SIMPLE continuity");
        hist.push_back(c0);
        rep->initial_continuity_rms = c0;
        rep->final_continuity_rms = c0;
    }
    if (!status) e = cudaEventRecord(e0, st);
    const int nfb = grid_for((long long)nfx + nfy);
    const FlursysLinearSolverOptions &mo = c.momentum_solver, &po = c.pressure_solver;
    for (long long it = 1; !status && it <= c.max_outer_iterations; ++it) {
        e = cudaMemsetAsync(flag, 0, sizeof(int), st);
        k_grad<<<ncb, kBlk, 0, st>>>(g, p, c.outlet_pressure, gx, gy);
        k_momentum<<<ncb, kBlk, 0, st>>>(g, Fx, Fy, gx, gy, u, v, mvals, bu, bv, rau, flag);
        if (e == cudaSuccess) e = cudaMemcpyAsync(us, u, 8.0 * n, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(vs, v, 8.0 * n, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess)
            e = csr_device_launch(2, n, d_ro, d_ci, mvals, bu, us, mo.absolute_tolerance, mo.relative_tolerance,
                                  mo.max_iterations, wu, st);
        if (e == cudaSuccess)
            e = csr_device_launch(2, n, d_ro, d_ci, mvals, bv, vs, mo.absolute_tolerance, mo.relative_tolerance,
                                  mo.max_iterations, wv, st);
        k_rhie_chow<<<nfb, kBlk, 0, st>>>(g, us, vs, p, gx, gy, rau, Fx, Fy, Fxp, Fyp, cfx, cfy);
        k_passemble<<<ncb, kBlk, 0, st>>>(g, Fxp, Fyp, cfx, cfy, pvals, prhs);
        if (e == cudaSuccess) e = cudaMemsetAsync(pc, 0, 8.0 * n, st);
        if (e == cudaSuccess)
            e = csr_device_launch(1, n, d_ro, d_ci, pvals, prhs, pc, po.absolute_tolerance, po.relative_tolerance,
                                  po.max_iterations, wp, st);
        k_grad<<<ncb, kBlk, 0, st>>>(g, pc, c.outlet_pressure, gx, gy);
        k_velocity<<<ncb, kBlk, 0, st>>>(n, c.pressure_relaxation, pc, p, us, vs, rau, gx, gy, u, v);
        k_flux<<<nfb, kBlk, 0, st>>>(g, Fxp, Fyp, cfx, cfy, pc, Fx, Fy);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(h_flag, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
        double cont = 0.0;
        if (e == cudaSuccess) e = continuity(&cont);
        if (e != cudaSuccess) { status = set_cuda_error(err, e, "SIMPLE outer iteration"); break; }
        if (*h_flag & 1) { status = fail(err, "backflow on a zero-gradient velocity boundary face", FLURSYS_ERR_INVALID_CONFIG); break; }
        if (*h_flag & 2) { status = fail(err, "invalid momentum diagonal", FLURSYS_ERR_BREAKDOWN); break; }
        if ((status = csr_device_status(wu.hres, &rep->momentum[0], err))) break;
        if ((status = csr_device_status(wv.hres, &rep->momentum[1], err))) break;
        if ((status = csr_device_status(wp.hres, &rep->pressure, err))) break;
        rep->momentum[2] = FlursysLinearSolveReport{FLURSYS_LINEAR_CONVERGED, 0, 0, 0.0, 0.0, 0.0};
        if (rep->momentum[0].status != FLURSYS_LINEAR_CONVERGED || rep->momentum[1].status != FLURSYS_LINEAR_CONVERGED) {
            status = fail(err, "momentum linear solve did not converge", FLURSYS_ERR_BREAKDOWN);
            break;
        }
        if (rep->pressure.status != FLURSYS_LINEAR_CONVERGED) {
            status = fail(err, "pressure-correction linear solve did not converge", FLURSYS_ERR_BREAKDOWN);
            break;
        }
        hist.push_back(cont);
        rep->outer_iterations = it;
        rep->final_continuity_rms = cont;
        if (cont <= c.continuity_tolerance) {
            rep->converged = 1;
            break;
        }
    }
    if (!status) {
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        rep->solve_ms = ms;
        std::vector<double> hfx(nfx), hfy(nfy);
        e = cudaMemcpyAsync(hfx.data(), Fx, 8 * nfx, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hfy.data(), Fy, 8 * nfy, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && hu) e = cudaMemcpyAsync(hu, u, 8.0 * n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && hv) e = cudaMemcpyAsync(hv, v, 8.0 * n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && hp) e = cudaMemcpyAsync(hp, p, 8.0 * n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            status = set_cuda_error(err, e, "SIMPLE results");
        } else {
            // backflow at the pressure outlet, boundary flux sums
            for (int j = 0; j < ny && !status; ++j)
                if (hfx[nx + (nx + 1) * j] < 0.0)
                    status = fail(err, "backflow at the pressure outlet", FLURSYS_ERR_INVALID_CONFIG);
            auto acc = [&](double owner_flux) {
                if (owner_flux < 0.0) rep->total_inflow += owner_flux;
                else rep->total_outflow += owner_flux;
            };
            for (int j = 0; j < ny; ++j) acc(-hfx[(nx + 1) * j]);
            for (int j = 0; j < ny; ++j) acc(hfx[nx + (nx + 1) * j]);
            for (int i = 0; i < nx; ++i) acc(-hfy[i]);
            for (int i = 0; i < nx; ++i) acc(hfy[i + nx * ny]);
            if (hflux) {
                std::memcpy(hflux, hfx.data(), 8 * nfx);
                std::memcpy(hflux + nfx, hfy.data(), 8 * nfy);
            }
            if (hhist) std::memcpy(hhist, hist.data(), 8 * hist.size());
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    wu.release();
    wv.release();
    wp.release();
    for (void *q : allocs) cudaFree(q);
    if (h_part) cudaFreeHost(h_part);
    if (h_flag) cudaFreeHost(h_flag);
    cudaStreamDestroy(st);
    return status;
}

}  // namespace flursys

using namespace flursys;

extern "C" int32_t flursys_cuda_simple_default_config(FlursysSimpleConfig *cfg) {
    if (!cfg) return FLURSYS_ERR_INVALID_ARGUMENT;
    std::memset(cfg, 0, sizeof *cfg);
    cfg->abi_version = FLURSYS_CUDA_ABI_VERSION;
    cfg->nx = 2048;
    cfg->ny = 512;
    cfg->length = 8.0;
    cfg->height = 1.0;
    cfg->inlet_peak_velocity = 1.0;
    cfg->kinematic_viscosity = (2.0 / 3.0) * 1.0 * 1.0 / 200.0;  // Re 200 on the mean velocity and the height
    cfg->outlet_pressure = 0.0;
    cfg->max_outer_iterations = 200;
    cfg->continuity_tolerance = 1.0e-10;
    cfg->velocity_relaxation = 0.7;
    cfg->pressure_relaxation = 0.3;
    cfg->momentum_solver = FlursysLinearSolverOptions{1.0e-10, 1.0e-8, 1000};
    cfg->pressure_solver = FlursysLinearSolverOptions{1.0e-10, 1.0e-8, 1000};
    return FLURSYS_OK;
}

extern "C" int32_t flursys_cuda_simple_channel(const FlursysSimpleConfig *cfg, double *velocity_x, double *velocity_y,
                                               double *pressure, double *face_flux, double *continuity_history,
                                               FlursysSimpleReport *report) {
    if (!cfg || !report) {
        set_global_error("simple_channel: null config or report");
        return FLURSYS_ERR_INVALID_ARGUMENT;
    }
    std::string err;
    const int32_t st = simple_channel_device(*cfg, velocity_x, velocity_y, pressure, face_flux, continuity_history,
                                             report, &err);
    if (st) set_global_error(err);
    return st;
}
