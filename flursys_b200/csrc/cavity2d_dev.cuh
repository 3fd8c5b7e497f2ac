// cavity2d_dev.cuh — per-element device functions of the 2D projection step,
// shared by the single-grid kernels (cavity2d.cu) and the batched ones
// (batch2d.cu).
#pragma once

#include <cuda_runtime.h>

#include "cavity2d.cuh"
#include "common.cuh"
#include "pcg2d.cuh"

namespace flursys {

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

// predict_momentum (:748-922) for face `id` of the concatenated u (nu) and
// v (nv) face sets; every face is written. The Boussinesq term
// g * beta * (T_face - T_ref) (:831-846, :896-911) is 0.0 when buoyancy is off.
__device__ __forceinline__ void predict_elem(const Cavity2dState &s, int id, double dt, int with_p, double relax) {
    const int nu = (s.nx + 1) * s.ny;
    const double *u = s.u, *v = s.v, *p = s.p;
    if (id < nu) {
        const int j = id / (s.nx + 1), i = id - j * (s.nx + 1);
        if (i == 0 || i == s.nx || !u_open(s, i, j)) { s.us[id] = 0.0; return; }
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
        const double bx = s.buoyancy ? s.gbx * (0.5 * (s.temp[i - 1 + s.nx * j] + s.temp[i + s.nx * j]) - s.tref) : 0.0;
        s.us[id] = up + relax * dt * (-conv + s.nu * diff - pg / s.rho + bx);
    } else {
        const int vid = id - nu;
        const int j = vid / s.nx, i = vid - j * s.nx;
        if (j == 0 || j == s.ny || !v_open(s, i, j)) { s.vs[vid] = 0.0; return; }
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
        const double by = s.buoyancy ? s.gby * (0.5 * (s.temp[i + s.nx * (j - 1)] + s.temp[i + s.nx * j]) - s.tref) : 0.0;
        s.vs[vid] = vp + relax * dt * (-conv + s.nu * diff - pg / s.rho + by);
    }
}

// apply_velocity_boundaries (:1981-2027) for row t of the left/right faces
// and column t of the bottom/top faces.
__device__ __forceinline__ void boundary_elem(const Cavity2dState &s, double *u, double *v, int t) {
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

// build_pressure_rhs (:924-970) for cell c
__device__ __forceinline__ void rhs_elem(const Cavity2dState &s, int c, double rho_over_dt) {
    if (s.flags[c] & 3) { s.rhs[c] = 0.0; return; }
    const int j = c / s.nx, i = c - j * s.nx;
    const double div = (s.us[i + 1 + (s.nx + 1) * j] - s.us[i + (s.nx + 1) * j]) / s.dx +
                       (s.vs[i + s.nx * (j + 1)] - s.vs[i + s.nx * j]) / s.dy;
    s.rhs[c] = rho_over_dt * div;
}

// correct_velocity (:1322-1379) for face `id` into (un, vn)
__device__ __forceinline__ void correct_elem(const Cavity2dState &s, int id, double dt_over_rho) {
    const int nu = (s.nx + 1) * s.ny;
    if (id < nu) {
        const int j = id / (s.nx + 1), i = id - j * (s.nx + 1);
        if (i == 0 || i == s.nx) { s.un[id] = s.us[id]; return; }
        s.un[id] = u_open(s, i, j) ? s.us[id] - dt_over_rho * ((s.p[i + s.nx * j] - s.p[i - 1 + s.nx * j]) / s.dx)
                                   : 0.0;
    } else {
        const int vid = id - nu;
        const int j = vid / s.nx, i = vid - j * s.nx;
        if (j == 0 || j == s.ny) { s.vn[vid] = s.vs[vid]; return; }
        s.vn[vid] = v_open(s, i, j) ? s.vs[vid] - dt_over_rho * ((s.p[i + s.nx * j] - s.p[i + s.nx * (j - 1)]) / s.dy)
                                    : 0.0;
    }
}

__device__ __forceinline__ double vcell(const Cavity2dState &s, int i, int j) {
    return 0.5 * (s.vn[i + s.nx * j] + s.vn[i + s.nx * (j + 1)]);
}
__device__ __forceinline__ double ucell(const Cavity2dState &s, int i, int j) {
    return 0.5 * (s.un[i + (s.nx + 1) * j] + s.un[i + 1 + (s.nx + 1) * j]);
}

// Running reductions of the post-step pass.
struct PostAcc {
    double mdiv = 0.0, mspeed = 0.0, mu = 0.0, mv = 0.0, du = 0.0, dv = 0.0, fx = 0.0, fy = 0.0;
    double muc = 0.0, mvc = 0.0;
};

// compute_cell_fields (:1381-1439), max_divergence (:1569-1582), the velocity
// maxima and changes of advance_one_step (:716-731), the finite scan of
// ensure_finite (:1707-1742) and the cylinder force sums (:1642-1668) for
// element `id` of max(cells, u faces, v faces).
__device__ __forceinline__ void post_elem(const Cavity2dState &s, int id, PostAcc &a) {
    const int nc = s.nx * s.ny, nu = (s.nx + 1) * s.ny, nv = s.nx * (s.ny + 1);
    if (id < nc) {
        const int j = id / s.nx, i = id - j * s.nx;
        if (sol(s, i, j)) {
            s.uc[id] = 0.0; s.vc[id] = 0.0; s.speed[id] = 0.0; s.vort[id] = 0.0;
        } else {
            const double uu = ucell(s, i, j), vv = vcell(s, i, j);
            const double sp = sqrt(uu * uu + vv * vv);
            s.uc[id] = uu; s.vc[id] = vv; s.speed[id] = sp;
            a.mspeed = fmax(a.mspeed, sp);
            a.muc = fmax(a.muc, fabs(uu));
            a.mvc = fmax(a.mvc, fabs(vv));
            if (!isfinite(sp)) atomicMin(&s.diag->bad_index[3], (unsigned long long)id);
            const bool e_ok = i + 1 < s.nx && !sol(s, i + 1, j), w_ok = i > 0 && !sol(s, i - 1, j);
            const bool n_ok = j + 1 < s.ny && !sol(s, i, j + 1), s_ok = j > 0 && !sol(s, i, j - 1);
            double dvdx = 0.0, dudy = 0.0;
            if (e_ok && w_ok) dvdx = (vcell(s, i + 1, j) - vcell(s, i - 1, j)) / (2.0 * s.dx);
            else if (e_ok) dvdx = (vcell(s, i + 1, j) - vv) / s.dx;
            else if (w_ok) dvdx = (vv - vcell(s, i - 1, j)) / s.dx;
            if (n_ok && s_ok) dudy = (ucell(s, i, j + 1) - ucell(s, i, j - 1)) / (2.0 * s.dy);
            else if (n_ok) dudy = (ucell(s, i, j + 1) - uu) / s.dy;
            else if (s_ok) dudy = (uu - ucell(s, i, j - 1)) / s.dy;
            s.vort[id] = dvdx - dudy;
            const double div = (s.un[i + 1 + (s.nx + 1) * j] - s.un[i + (s.nx + 1) * j]) / s.dx +
                               (s.vn[i + s.nx * (j + 1)] - s.vn[i + s.nx * j]) / s.dy;
            a.mdiv = fmax(a.mdiv, fabs(div));
            if (s.cylinder) {
                const double pp = s.p[id];
                if (i + 1 < s.nx && sol(s, i + 1, j)) { a.fx += pp * s.dy; a.fy += s.cylinder_mu * vv / (0.5 * s.dx) * s.dy; }
                if (i > 0 && sol(s, i - 1, j)) { a.fx -= pp * s.dy; a.fy += s.cylinder_mu * vv / (0.5 * s.dx) * s.dy; }
                if (j + 1 < s.ny && sol(s, i, j + 1)) { a.fy += pp * s.dx; a.fx += s.cylinder_mu * uu / (0.5 * s.dy) * s.dx; }
                if (j > 0 && sol(s, i, j - 1)) { a.fy -= pp * s.dx; a.fx += s.cylinder_mu * uu / (0.5 * s.dy) * s.dx; }
            }
        }
        if (!isfinite(s.p[id])) atomicMin(&s.diag->bad_index[0], (unsigned long long)id);
    }
    if (id < nu) {
        const double x = s.un[id];
        a.mu = fmax(a.mu, fabs(x));
        a.du = fmax(a.du, fabs(x - s.u[id]));
        if (!isfinite(x)) atomicMin(&s.diag->bad_index[1], (unsigned long long)id);
    }
    if (id < nv) {
        const double x = s.vn[id];
        a.mv = fmax(a.mv, fabs(x));
        a.dv = fmax(a.dv, fabs(x - s.v[id]));
        if (!isfinite(x)) atomicMin(&s.diag->bad_index[2], (unsigned long long)id);
    }
}

// temperature_neighbor (:1495-1530): a solid neighbour or an adiabatic wall
// mirrors the centre; a fixed-temperature wall gives 2 T_w - centre.
__device__ __forceinline__ double temp_nb(const Cavity2dState &s, int i, int j, int di, int dj, double c) {
    const int ni = i + di, nj = j + dj;
    if (ni >= 0 && ni < s.nx && nj >= 0 && nj < s.ny) return sol(s, ni, nj) ? c : s.temp[ni + s.nx * nj];
    const int side = ni < 0 ? 0 : (ni >= s.nx ? 1 : (nj < 0 ? 2 : 3));
    return s.tkind[side] == FLURSYS_THERMAL_FIXED_TEMPERATURE ? 2.0 * s.twall[side] - c : c;
}

// advance_temperature (:1441-1493) for cell c: explicit conservative update
// with first-order upwind face values on the corrected face velocities.
__device__ __forceinline__ void temperature_elem(const Cavity2dState &s, int c, double dt) {
    const int j = c / s.nx, i = c - j * s.nx;
    const double ctr = s.temp[c];
    double t = ctr;
    if (!sol(s, i, j)) {
        const double e = temp_nb(s, i, j, 1, 0, ctr), w = temp_nb(s, i, j, -1, 0, ctr);
        const double n = temp_nb(s, i, j, 0, 1, ctr), so = temp_nb(s, i, j, 0, -1, ctr);
        const double ue = s.un[i + 1 + (s.nx + 1) * j], uw = s.un[i + (s.nx + 1) * j];
        const double vn = s.vn[i + s.nx * (j + 1)], vsf = s.vn[i + s.nx * j];
        const double fe = ue * (ue >= 0.0 ? ctr : e), fw = uw * (uw >= 0.0 ? w : ctr);
        const double fn = vn * (vn >= 0.0 ? ctr : n), fs = vsf * (vsf >= 0.0 ? so : ctr);
        const double conv = (fe - fw) / s.dx + (fn - fs) / s.dy;
        const double diff = (e - 2.0 * ctr + w) / (s.dx * s.dx) + (n - 2.0 * ctr + so) / (s.dy * s.dy);
        t = ctr + dt * (-conv + s.alpha * diff + s.tsource);
    }
    s.temp_next[c] = t;
    if (!isfinite(t)) atomicMin(&s.diag->bad_index[4], (unsigned long long)c);
}

}  // namespace flursys
