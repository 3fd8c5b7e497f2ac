// flursys_oracle.cpp — TEST INFRASTRUCTURE ONLY: the CPU FP64 oracle.
//
// A restatement, in C++17, of the FLURSYS reference algorithms on the
// structured MAC projection path and of src/linear. Each function cites the
// reference file:line it follows (paths relative to the FLURSYS tree). It is
// used only by tests/ (as the checker), by __graft_entry__.smoke() and by
// bench.py's CPU baseline; the CUDA product library never links it.
//
// Reduction order: with orc_set_threads(1) every sum is serial left to right.
// The reference reduces on a Rayon pool; its own test pins 1-vs-4-thread
// results only to 1e-10 (tests/smoke.rs:132-155), so reduction order is a
// rounding-level effect here too.
#include "flursys_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <tuple>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

int g_threads = 1;

void copy_msg(const std::string &s, char *buf, size_t size) {
    if (!buf || size == 0) return;
    size_t n = std::min(size - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = '\0';
}

// Rust's `{:.Ne}` formatting of an f64: mantissa with N decimals, then `e`
// and the exponent without sign padding or leading zeros ("1.500e-5").
std::string rust_sci(double v, int prec) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.*e", prec, v);
    std::string s(buf);
    const size_t e = s.find('e');
    if (e == std::string::npos) return s;
    const std::string mant = s.substr(0, e);
    int exp10 = std::atoi(s.c_str() + e + 1);
    return mant + "e" + std::to_string(exp10);
}

// ---------------------------------------------------------------------------
// Vector primitives (src/linear/vector.rs and the Rayon helpers of
// incompressible.rs:1308-1320).
// ---------------------------------------------------------------------------
double dot(const std::vector<double> &a, const std::vector<double> &b) {
    const int64_t n = (int64_t)a.size();
    double s = 0.0;
    if (g_threads <= 1) {
        for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    } else {
#pragma omp parallel for reduction(+ : s) num_threads(g_threads) schedule(static)
        for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    }
    return s;
}

double max_abs(const std::vector<double> &a) {
    const int64_t n = (int64_t)a.size();
    double m = 0.0;
    if (g_threads <= 1) {
        for (int64_t i = 0; i < n; ++i) m = std::max(m, std::fabs(a[i]));
    } else {
#pragma omp parallel for reduction(max : m) num_threads(g_threads) schedule(static)
        for (int64_t i = 0; i < n; ++i) m = std::max(m, std::fabs(a[i]));
    }
    return m;
}

// Field2D::max_abs (field.rs:49-51): fold with f64::max, which ignores NaN
// exactly as std::max(m, x) does with a NaN second argument.
double field_max_abs(const std::vector<double> &a) {
    double m = 0.0;
    for (double x : a) m = std::max(m, std::fabs(x));
    return m;
}

bool all_finite(const std::vector<double> &a, size_t *bad) {
    for (size_t i = 0; i < a.size(); ++i)
        if (!std::isfinite(a[i])) {
            if (bad) *bad = i;
            return false;
        }
    return true;
}

// ---------------------------------------------------------------------------
// Shared matrix-free PCG core. It follows the iteration order of
// solve_pressure_pcg (incompressible.rs:1048-1214): initial residual and test,
// Jacobi z, d = z, loop { q = A d; dq; alpha; x += a d; r -= a q; residual;
// test; z; rz_new; beta; d = z + beta d }. Zero-mean projections
// (project_zero_mean, :2338-2377) run where the reference runs them when the
// operator is pure Neumann.
// ---------------------------------------------------------------------------
struct StructuredOperator {
    // Returns true when the row is an identity row (solid, outlet, pinned cell).
    virtual bool identity_row(int64_t k) const = 0;
    virtual void apply(const std::vector<double> &x, std::vector<double> &y) const = 0;
    virtual double diagonal(int64_t k) const = 0;  // 0 for identity rows
    virtual bool needs_projection() const = 0;
    virtual void project(std::vector<double> &v) const = 0;
    virtual ~StructuredOperator() = default;
};

struct PcgResult {
    int32_t status = FLURSYS_OK;
    int32_t linear_status = FLURSYS_LINEAR_CONVERGED;
    int64_t iterations = 0;
    double initial = 0.0;
    double residual = 0.0;
    std::string error;
};

struct StopRule {
    int32_t rule = FLURSYS_STOP_ABS_INF;
    double tol = 1e-5;   // ABS_INF / REFERENCE_RESIDUAL
    double atol = 0.0;   // REL_L2
    double rtol = 1e-8;  // REL_L2
    double threshold = 0.0;
    double norm(const std::vector<double> &r) const {
        return rule == FLURSYS_STOP_REL_L2 ? std::sqrt(dot(r, r)) : max_abs(r);
    }
    void set_initial(double r0) {
        threshold = rule == FLURSYS_STOP_REL_L2 ? atol + rtol * r0 : tol;
    }
    // ABS_INF keeps the strict `<` of incompressible.rs:1112,1162; REL_L2 the
    // `<=` of src/linear/solver.rs:86,115.
    bool done(double res) const {
        return rule == FLURSYS_STOP_REL_L2 ? res <= threshold : res < threshold;
    }
};

PcgResult pcg_core(const StructuredOperator &op, const std::vector<double> &b_in,
                   std::vector<double> &x, StopRule stop, int64_t max_iters) {
    const int64_t n = (int64_t)x.size();
    std::vector<double> b(b_in), r(n), z(n), d(n), q(n);
    PcgResult res;
    const bool proj = op.needs_projection();
    auto jacobi = [&](const std::vector<double> &rr, std::vector<double> &zz) {
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
        for (int64_t k = 0; k < n; ++k) {
            double dg = op.diagonal(k);
            zz[k] = (op.identity_row(k) || !(dg > 0.0)) ? rr[k] : rr[k] / dg;
        }
    };
    if (proj) {
        op.project(x);
        op.project(b);
    }
    op.apply(x, q);
    for (int64_t k = 0; k < n; ++k) r[k] = b[k] - q[k];
    if (proj) op.project(r);
    double residual = stop.norm(r);
    res.initial = residual;
    stop.set_initial(residual);
    if (stop.done(residual)) {
        res.residual = residual;
        return res;
    }
    jacobi(r, z);
    if (proj) op.project(z);
    d = z;
    double rz_old = dot(r, z);
    int64_t iterations = 0;
    bool converged = false;
    for (int64_t it = 0; it < max_iters; ++it) {
        iterations = it + 1;
        op.apply(d, q);
        double den = dot(d, q);
        if (std::fabs(den) < 1.0e-30 || !std::isfinite(den)) {
            res.status = FLURSYS_ERR_BREAKDOWN;
            res.error = "PCG pressure solver encountered a singular search direction";
            return res;
        }
        double alpha = rz_old / den;
        if (!std::isfinite(alpha)) {
            res.status = FLURSYS_ERR_BREAKDOWN;
            res.error = "PCG pressure solver produced a non-finite step length";
            return res;
        }
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
        for (int64_t k = 0; k < n; ++k) {
            x[k] += alpha * d[k];
            r[k] -= alpha * q[k];
        }
        if (proj) {
            op.project(x);
            op.project(r);
        }
        residual = stop.norm(r);
        if (!std::isfinite(residual)) {
            res.status = FLURSYS_ERR_NON_FINITE;
            res.error = "PCG pressure solver produced a non-finite residual";
            return res;
        }
        if (stop.done(residual)) {
            converged = true;
            break;
        }
        jacobi(r, z);
        if (proj) op.project(z);
        double rz_new = dot(r, z);
        if (std::fabs(rz_old) < 1.0e-30) break;
        double beta = rz_new / rz_old;
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
        for (int64_t k = 0; k < n; ++k) d[k] = z[k] + beta * d[k];
        if (proj) op.project(d);
        rz_old = rz_new;
    }
    res.iterations = iterations;
    res.residual = residual;
    res.linear_status = converged ? FLURSYS_LINEAR_CONVERGED : FLURSYS_LINEAR_MAX_ITERATIONS;
    return res;
}

// ---------------------------------------------------------------------------
// 3D pinned Neumann operator: the system that the 3D SOR converges to
// (incompressible_3d.rs:293-332, pressure_neighbor :450-474). For cells other
// than (0,0,0): (A x)_c = sum_{in-range nb} w (x_c - x_nb) with x_(0,0,0) = 0;
// cell (0,0,0) is an identity row. A x = -rhs is Lap(p) = rhs with p pinned.
// ---------------------------------------------------------------------------
struct Pinned3DOperator final : StructuredOperator {
    int64_t nx, ny, nz;
    double ix2, iy2, iz2;
    Pinned3DOperator(int64_t nx_, int64_t ny_, int64_t nz_, double dx, double dy, double dz)
        : nx(nx_), ny(ny_), nz(nz_), ix2(1.0 / (dx * dx)), iy2(1.0 / (dy * dy)),
          iz2(1.0 / (dz * dz)) {}
    bool identity_row(int64_t k) const override { return k == 0; }
    double diagonal(int64_t k) const override {
        if (k == 0) return 0.0;
        int64_t i = k % nx, j = (k / nx) % ny, kk = k / (nx * ny);
        double dg = 0.0;
        if (i + 1 < nx) dg += ix2;
        if (i > 0) dg += ix2;
        if (j + 1 < ny) dg += iy2;
        if (j > 0) dg += iy2;
        if (kk + 1 < nz) dg += iz2;
        if (kk > 0) dg += iz2;
        return dg;
    }
    void apply(const std::vector<double> &x, std::vector<double> &y) const override {
        const int64_t sxy = nx * ny;
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
        for (int64_t kk = 0; kk < nz; ++kk)
            for (int64_t j = 0; j < ny; ++j)
                for (int64_t i = 0; i < nx; ++i) {
                    int64_t c = i + nx * (j + ny * kk);
                    if (c == 0) {
                        y[c] = x[c];
                        continue;
                    }
                    double dg = 0.0, s = 0.0;
                    if (i + 1 < nx) { dg += ix2; s += ix2 * (c + 1 == 0 ? 0.0 : x[c + 1]); }
                    if (i > 0) { dg += ix2; s += ix2 * (c - 1 == 0 ? 0.0 : x[c - 1]); }
                    if (j + 1 < ny) { dg += iy2; s += iy2 * x[c + nx]; }
                    if (j > 0) { dg += iy2; s += iy2 * (c - nx == 0 ? 0.0 : x[c - nx]); }
                    if (kk + 1 < nz) { dg += iz2; s += iz2 * x[c + sxy]; }
                    if (kk > 0) { dg += iz2; s += iz2 * (c - sxy == 0 ? 0.0 : x[c - sxy]); }
                    y[c] = dg * x[c] - s;
                }
    }
    bool needs_projection() const override { return false; }
    void project(std::vector<double> &) const override {}
};

// ---------------------------------------------------------------------------
// Case data (src/cases/mod.rs:120-227, cavity.rs, channel.rs, cylinder.rs,
// backward_step.rs) and boundary overrides (src/preprocess.rs:1362-1406).
// ---------------------------------------------------------------------------
enum BKind { BK_VELOCITY = 0, BK_SYMMETRY = 1, BK_OUTLET = 2 };

struct CaseModel {
    FlursysCaseParams c;
    FlursysBoundaryOverride ov[4];

    // Case::boundary_kind (mod.rs:120-139)
    BKind case_kind(int side, double *outlet_p) const {
        *outlet_p = 0.0;
        switch (c.kind) {
            case FLURSYS_CASE_CAVITY: return BK_VELOCITY;
            case FLURSYS_CASE_CYLINDER:
                if (side == FLURSYS_SIDE_LEFT) return BK_VELOCITY;
                if (side == FLURSYS_SIDE_RIGHT) return BK_OUTLET;
                return BK_SYMMETRY;
            default:  // backward step, channel
                if (side == FLURSYS_SIDE_RIGHT) return BK_OUTLET;
                return BK_VELOCITY;
        }
    }
    // SolverBoundaryOverrides::kind (preprocess.rs:1370-1379)
    BKind kind(int side, double *outlet_p = nullptr) const {
        double dummy;
        double *op = outlet_p ? outlet_p : &dummy;
        switch (ov[side].kind) {
            case FLURSYS_BOUNDARY_VELOCITY: *op = 0.0; return BK_VELOCITY;
            case FLURSYS_BOUNDARY_PRESSURE_OUTLET: *op = ov[side].pressure; return BK_OUTLET;
            case FLURSYS_BOUNDARY_SYMMETRY: *op = 0.0; return BK_SYMMETRY;
            default: return case_kind(side, op);
        }
    }
    // Case::boundary_velocity (mod.rs:142-175)
    void case_velocity(int side, double /*x*/, double y, double *u, double *v) const {
        *u = 0.0;
        *v = 0.0;
        switch (c.kind) {
            case FLURSYS_CASE_CAVITY:
                if (side == FLURSYS_SIDE_TOP) *u = c.reference_velocity;
                return;
            case FLURSYS_CASE_CYLINDER: *u = c.reference_velocity; return;
            case FLURSYS_CASE_BACKWARD_STEP:
                if (side == FLURSYS_SIDE_LEFT) {
                    if (y <= c.step_height) return;
                    double inlet = c.height - c.step_height;
                    double eta = std::clamp((y - c.step_height) / inlet, 0.0, 1.0);
                    *u = 6.0 * c.reference_velocity * eta * (1.0 - eta);
                } else if (side == FLURSYS_SIDE_RIGHT) {
                    *u = c.reference_velocity;
                }
                return;
            default:  // channel
                if (side == FLURSYS_SIDE_LEFT) {
                    double eta = std::clamp(y / c.height, 0.0, 1.0);
                    *u = 6.0 * c.reference_velocity * eta * (1.0 - eta);
                } else if (side == FLURSYS_SIDE_RIGHT) {
                    *u = c.reference_velocity;
                }
                return;
        }
    }
    // SolverBoundaryOverrides::velocity (preprocess.rs:1381-1388)
    void velocity(int side, double x, double y, double *u, double *v) const {
        switch (ov[side].kind) {
            case FLURSYS_BOUNDARY_VELOCITY: *u = ov[side].u; *v = ov[side].v; return;
            case FLURSYS_BOUNDARY_PRESSURE_OUTLET:
            case FLURSYS_BOUNDARY_SYMMETRY: *u = 0.0; *v = 0.0; return;
            default: case_velocity(side, x, y, u, v);
        }
    }
    // Case::initial_velocity (mod.rs:177-216)
    void initial_velocity(double x, double y, double *u, double *v) const {
        *u = 0.0;
        *v = 0.0;
        switch (c.kind) {
            case FLURSYS_CASE_CAVITY: return;
            case FLURSYS_CASE_CYLINDER: {
                double r2 = (x - c.cylinder_xc) * (x - c.cylinder_xc) +
                            (y - c.cylinder_yc) * (y - c.cylinder_yc);
                double rad = 0.5 * c.cylinder_diameter;
                if (r2 <= rad * rad) return;
                double xp = c.cylinder_xc + 1.5 * c.cylinder_diameter;
                double yp = c.cylinder_yc + 0.25 * c.cylinder_diameter;
                double sigma2 = c.cylinder_diameter * c.cylinder_diameter;
                double ddx = x - xp, ddy = y - yp;
                double psi = c.cylinder_perturbation * std::exp(-(ddx * ddx + ddy * ddy) / sigma2);
                *u = c.reference_velocity + (-2.0 * ddy / sigma2 * psi);
                *v = 2.0 * ddx / sigma2 * psi;
                return;
            }
            case FLURSYS_CASE_BACKWARD_STEP:
                if (x < c.step_x && y < c.step_height) return;
                if (y > c.step_height) {
                    double inlet = c.height - c.step_height;
                    double eta = std::clamp((y - c.step_height) / inlet, 0.0, 1.0);
                    *u = 6.0 * c.reference_velocity * eta * (1.0 - eta);
                } else {
                    *u = c.reference_velocity;
                }
                return;
            default: {
                double eta = std::clamp(y / c.height, 0.0, 1.0);
                *u = 6.0 * c.reference_velocity * eta * (1.0 - eta);
                return;
            }
        }
    }
    // Case::is_solid (mod.rs:218-227)
    bool is_solid(double x, double y) const {
        switch (c.kind) {
            case FLURSYS_CASE_CYLINDER: {
                double rad = 0.5 * c.cylinder_diameter;
                return (x - c.cylinder_xc) * (x - c.cylinder_xc) +
                           (y - c.cylinder_yc) * (y - c.cylinder_yc) <=
                       rad * rad;
            }
            case FLURSYS_CASE_BACKWARD_STEP: return x < c.step_x && y < c.step_height;
            default: return false;
        }
    }
};

// ---------------------------------------------------------------------------
// adaptive_time_step (incompressible.rs:2308-2336) and
// momentum_stability_numbers (:2294-2306).
// ---------------------------------------------------------------------------
int32_t adaptive_dt(double current_dt, double mu, double mv, double dx, double dy, double nu,
                    double alpha_thermal, double min_dt, double max_dt, double target_cfl,
                    double target_diff, double growth, double *out, std::string *err) {
    double advective_rate = mu / dx + mv / dy;
    double cfl_dt = advective_rate > 2.220446049250313e-16 ? target_cfl / advective_rate : max_dt;
    double inv = 1.0 / (dx * dx) + 1.0 / (dy * dy);
    double eff = alpha_thermal >= 0.0 ? std::max(alpha_thermal, nu) : nu;
    double diffusion_dt = target_diff / (eff * inv);
    double stable = std::min(std::min(max_dt, cfl_dt), diffusion_dt);
    if (stable < min_dt) {
        if (err)
            *err = "required stable time step " + rust_sci(stable, 3) + " is below configured min_dt " +
                   rust_sci(min_dt, 3) + "; CFL constraint=" + rust_sci(cfl_dt, 3) +
                   ", diffusion constraint=" + rust_sci(diffusion_dt, 3);
        return FLURSYS_ERR_INVALID_CONFIG;
    }
    double limited = std::min(stable, current_dt * growth);
    *out = std::clamp(limited, min_dt, max_dt);
    return FLURSYS_OK;
}

// ---------------------------------------------------------------------------
// Solver base.
// ---------------------------------------------------------------------------
}  // namespace

struct OracleSolver {
    FlursysCudaConfig cfg{};
    std::string err;
    int64_t step = 0;
    double time = 0.0;
    virtual ~OracleSolver() = default;
    virtual int32_t advance(FlursysStepReport *rep) = 0;
    virtual std::vector<double> *field(int32_t id) = 0;
    virtual int32_t predict(double dt) = 0;
    virtual int32_t rhs_phase(double dt) = 0;
    virtual int32_t pressure(double *res, int64_t *its) = 0;
    virtual int32_t correct(double dt) = 0;
    virtual double max_divergence() const = 0;
    virtual double pressure_residual() const = 0;
    virtual double max_speed() const = 0;
};

namespace {

// ---------------------------------------------------------------------------
// 3D: LidDrivenCavity3DSolver (incompressible_3d.rs).
// ---------------------------------------------------------------------------
struct Solver3D final : OracleSolver {
    int64_t nx, ny, nz;
    double dx, dy, dz, nu, lid, rho, dt;
    std::vector<double> p, rhs, u, v, w, us, vs, ws;

    size_t iu(int64_t i, int64_t j, int64_t k) const { return i + (nx + 1) * (j + ny * k); }
    size_t iv(int64_t i, int64_t j, int64_t k) const { return i + nx * (j + (ny + 1) * k); }
    size_t iw(int64_t i, int64_t j, int64_t k) const { return i + nx * (j + ny * k); }
    size_t ic(int64_t i, int64_t j, int64_t k) const { return i + nx * (j + ny * k); }

    explicit Solver3D(const FlursysCudaConfig &c) {
        cfg = c;
        nx = c.nx; ny = c.ny; nz = c.nz;
        dx = c.case_params.length / nx;
        dy = c.case_params.height / ny;
        dz = c.case_params.depth / nz;
        lid = c.case_params.reference_velocity;
        rho = c.case_params.density;
        nu = lid * c.case_params.length / c.case_params.reynolds;  // viscosity() :86-88
        dt = c.dt;
        size_t nc = nx * ny * nz;
        p.assign(nc, 0.0);
        rhs.assign(nc, 0.0);
        u.assign((nx + 1) * ny * nz, 0.0);
        v.assign(nx * (ny + 1) * nz, 0.0);
        w.assign(nx * ny * (nz + 1), 0.0);
        us = u; vs = v; ws = w;
    }

    // u_neighbor / v_neighbor / w_neighbor (:365-447)
    double u_nb(int64_t i, int64_t j, int64_t k, int di, int dj, int dk, double c) const {
        int64_t ni = i + di, nj = j + dj, nk = k + dk;
        if (ni >= 0 && ni <= nx && nj >= 0 && nj < ny && nk >= 0 && nk < nz) return u[iu(ni, nj, nk)];
        return nj >= ny ? 2.0 * lid - c : -c;
    }
    double v_nb(int64_t i, int64_t j, int64_t k, int di, int dj, int dk, double c) const {
        int64_t ni = i + di, nj = j + dj, nk = k + dk;
        if (ni >= 0 && ni < nx && nj >= 0 && nj <= ny && nk >= 0 && nk < nz) return v[iv(ni, nj, nk)];
        return -c;
    }
    double w_nb(int64_t i, int64_t j, int64_t k, int di, int dj, int dk, double c) const {
        int64_t ni = i + di, nj = j + dj, nk = k + dk;
        if (ni >= 0 && ni < nx && nj >= 0 && nj < ny && nk >= 0 && nk <= nz) return w[iw(ni, nj, nk)];
        return -c;
    }
    double p_nb(int64_t i, int64_t j, int64_t k, int di, int dj, int dk, double c) const {
        int64_t ni = i + di, nj = j + dj, nk = k + dk;
        if (ni >= 0 && ni < nx && nj >= 0 && nj < ny && nk >= 0 && nk < nz) return p[ic(ni, nj, nk)];
        return c;
    }

    // predict_momentum (:174-273)
    int32_t predict(double step_dt) override {
        std::fill(us.begin(), us.end(), 0.0);
        std::fill(vs.begin(), vs.end(), 0.0);
        std::fill(ws.begin(), ws.end(), 0.0);
        const double dx2 = dx * dx, dy2 = dy * dy, dz2 = dz * dz;
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
        for (int64_t k = 0; k < nz; ++k)
            for (int64_t j = 0; j < ny; ++j)
                for (int64_t i = 1; i < nx; ++i) {
                    double c = u[iu(i, j, k)];
                    double e = u_nb(i, j, k, 1, 0, 0, c), wst = u_nb(i, j, k, -1, 0, 0, c);
                    double n = u_nb(i, j, k, 0, 1, 0, c), s = u_nb(i, j, k, 0, -1, 0, c);
                    double f = u_nb(i, j, k, 0, 0, 1, c), b = u_nb(i, j, k, 0, 0, -1, c);
                    double vb = 0.25 * (v[iv(i - 1, j, k)] + v[iv(i, j, k)] + v[iv(i - 1, j + 1, k)] +
                                        v[iv(i, j + 1, k)]);
                    double wb = 0.25 * (w[iw(i - 1, j, k)] + w[iw(i, j, k)] + w[iw(i - 1, j, k + 1)] +
                                        w[iw(i, j, k + 1)]);
                    us[iu(i, j, k)] =
                        c + step_dt * (-c * (e - wst) / (2.0 * dx) - vb * (n - s) / (2.0 * dy) -
                                       wb * (f - b) / (2.0 * dz) +
                                       nu * ((e - 2.0 * c + wst) / dx2 + (n - 2.0 * c + s) / dy2 +
                                             (f - 2.0 * c + b) / dz2));
                }
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
        for (int64_t k = 0; k < nz; ++k)
            for (int64_t j = 1; j < ny; ++j)
                for (int64_t i = 0; i < nx; ++i) {
                    double c = v[iv(i, j, k)];
                    double e = v_nb(i, j, k, 1, 0, 0, c), wst = v_nb(i, j, k, -1, 0, 0, c);
                    double n = v_nb(i, j, k, 0, 1, 0, c), s = v_nb(i, j, k, 0, -1, 0, c);
                    double f = v_nb(i, j, k, 0, 0, 1, c), b = v_nb(i, j, k, 0, 0, -1, c);
                    double ub = 0.25 * (u[iu(i, j - 1, k)] + u[iu(i + 1, j - 1, k)] + u[iu(i, j, k)] +
                                        u[iu(i + 1, j, k)]);
                    double wb = 0.25 * (w[iw(i, j - 1, k)] + w[iw(i, j, k)] + w[iw(i, j - 1, k + 1)] +
                                        w[iw(i, j, k + 1)]);
                    vs[iv(i, j, k)] =
                        c + step_dt * (-ub * (e - wst) / (2.0 * dx) - c * (n - s) / (2.0 * dy) -
                                       wb * (f - b) / (2.0 * dz) +
                                       nu * ((e - 2.0 * c + wst) / dx2 + (n - 2.0 * c + s) / dy2 +
                                             (f - 2.0 * c + b) / dz2));
                }
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
        for (int64_t k = 1; k < nz; ++k)
            for (int64_t j = 0; j < ny; ++j)
                for (int64_t i = 0; i < nx; ++i) {
                    double c = w[iw(i, j, k)];
                    double e = w_nb(i, j, k, 1, 0, 0, c), wst = w_nb(i, j, k, -1, 0, 0, c);
                    double n = w_nb(i, j, k, 0, 1, 0, c), s = w_nb(i, j, k, 0, -1, 0, c);
                    double f = w_nb(i, j, k, 0, 0, 1, c), b = w_nb(i, j, k, 0, 0, -1, c);
                    double ub = 0.25 * (u[iu(i, j, k - 1)] + u[iu(i + 1, j, k - 1)] + u[iu(i, j, k)] +
                                        u[iu(i + 1, j, k)]);
                    double vb = 0.25 * (v[iv(i, j, k - 1)] + v[iv(i, j + 1, k - 1)] + v[iv(i, j, k)] +
                                        v[iv(i, j + 1, k)]);
                    ws[iw(i, j, k)] =
                        c + step_dt * (-ub * (e - wst) / (2.0 * dx) - vb * (n - s) / (2.0 * dy) -
                                       c * (f - b) / (2.0 * dz) +
                                       nu * ((e - 2.0 * c + wst) / dx2 + (n - 2.0 * c + s) / dy2 +
                                             (f - 2.0 * c + b) / dz2));
                }
        return FLURSYS_OK;
    }

    // build_pressure_rhs (:275-291)
    int32_t rhs_phase(double step_dt) override {
        const double scale = rho / step_dt;
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
        for (int64_t k = 0; k < nz; ++k)
            for (int64_t j = 0; j < ny; ++j)
                for (int64_t i = 0; i < nx; ++i)
                    rhs[ic(i, j, k)] = scale * (us[iu(i + 1, j, k)] - us[iu(i, j, k)]) / dx +
                                       scale * (vs[iv(i, j + 1, k)] - vs[iv(i, j, k)]) / dy +
                                       scale * (ws[iw(i, j, k + 1)] - ws[iw(i, j, k)]) / dz;
        rhs[0] = 0.0;
        return FLURSYS_OK;
    }

    // pressure_residual (:476-502)
    double pressure_residual() const override {
        const double ix2 = 1.0 / (dx * dx), iy2 = 1.0 / (dy * dy), iz2 = 1.0 / (dz * dz);
        double m = 0.0;
        for (int64_t k = 0; k < nz; ++k)
            for (int64_t j = 0; j < ny; ++j)
                for (int64_t i = 0; i < nx; ++i) {
                    if (i == 0 && j == 0 && k == 0) continue;
                    double c = p[ic(i, j, k)];
                    double lap = ix2 * (p_nb(i, j, k, 1, 0, 0, c) - 2.0 * c + p_nb(i, j, k, -1, 0, 0, c)) +
                                 iy2 * (p_nb(i, j, k, 0, 1, 0, c) - 2.0 * c + p_nb(i, j, k, 0, -1, 0, c)) +
                                 iz2 * (p_nb(i, j, k, 0, 0, 1, c) - 2.0 * c + p_nb(i, j, k, 0, 0, -1, c));
                    // f64::max ignores NaN, as std::max(m, a) does here.
                    m = std::max(m, std::fabs(lap - rhs[ic(i, j, k)]));
                }
        return m;
    }

    // solve_pressure_poisson (:293-332): lexicographic SOR, p(0,0,0) = 0.
    int32_t pressure_sor(double *res_out, int64_t *its_out) {
        const double ix2 = 1.0 / (dx * dx), iy2 = 1.0 / (dy * dy), iz2 = 1.0 / (dz * dz);
        const double diag = 2.0 * (ix2 + iy2 + iz2);
        const double omega = cfg.pressure_omega;
        double residual = INFINITY;
        int64_t its = 0;
        for (int64_t it = 0; it < cfg.pressure_max_iters; ++it) {
            its = it + 1;
            for (int64_t k = 0; k < nz; ++k)
                for (int64_t j = 0; j < ny; ++j)
                    for (int64_t i = 0; i < nx; ++i) {
                        if (i == 0 && j == 0 && k == 0) {
                            p[0] = 0.0;
                            continue;
                        }
                        double c = p[ic(i, j, k)];
                        double s = ix2 * (p_nb(i, j, k, 1, 0, 0, c) + p_nb(i, j, k, -1, 0, 0, c)) +
                                   iy2 * (p_nb(i, j, k, 0, 1, 0, c) + p_nb(i, j, k, 0, -1, 0, c)) +
                                   iz2 * (p_nb(i, j, k, 0, 0, 1, c) + p_nb(i, j, k, 0, 0, -1, c));
                        double cand = (s - rhs[ic(i, j, k)]) / diag;
                        p[ic(i, j, k)] += omega * (cand - p[ic(i, j, k)]);
                    }
            residual = pressure_residual();
            if (!std::isfinite(residual)) {
                err = "3D pressure solver produced a non-finite residual";
                return FLURSYS_ERR_NON_FINITE;
            }
            if (residual < cfg.pressure_tolerance) break;
        }
        *res_out = residual;
        *its_out = its;
        return FLURSYS_OK;
    }

    int32_t pressure(double *res_out, int64_t *its_out) override {
        if (cfg.pressure_solver == FLURSYS_PRESSURE_SOR) return pressure_sor(res_out, its_out);
        // Jacobi-PCG on the same pinned system (the 3D configs name PCG).
        Pinned3DOperator op(nx, ny, nz, dx, dy, dz);
        std::vector<double> b(rhs.size());
        for (size_t k = 0; k < b.size(); ++k) b[k] = -rhs[k];
        b[0] = 0.0;
        std::vector<double> x(p);
        x[0] = 0.0;
        StopRule stop;
        stop.rule = cfg.stop_rule == FLURSYS_STOP_REL_L2 ? FLURSYS_STOP_REL_L2 : FLURSYS_STOP_ABS_INF;
        stop.tol = cfg.pressure_tolerance;
        stop.atol = cfg.pressure_atol;
        stop.rtol = cfg.pressure_rtol;
        PcgResult r = pcg_core(op, b, x, stop, cfg.pressure_max_iters);
        if (r.status != FLURSYS_OK) {
            err = r.error;
            return r.status;
        }
        p = x;
        last_initial = r.initial;
        last_linear_status = r.linear_status;
        *res_out = r.residual;
        *its_out = r.iterations;
        return FLURSYS_OK;
    }
    double last_initial = 0.0;
    int32_t last_linear_status = FLURSYS_LINEAR_CONVERGED;

    // correct_velocity (:334-363)
    int32_t correct(double step_dt) override {
        const double scale = step_dt / rho;
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
        for (int64_t k = 0; k < nz; ++k) {
            for (int64_t j = 0; j < ny; ++j)
                for (int64_t i = 1; i < nx; ++i)
                    u[iu(i, j, k)] = us[iu(i, j, k)] - scale * (p[ic(i, j, k)] - p[ic(i - 1, j, k)]) / dx;
            for (int64_t j = 1; j < ny; ++j)
                for (int64_t i = 0; i < nx; ++i)
                    v[iv(i, j, k)] = vs[iv(i, j, k)] - scale * (p[ic(i, j, k)] - p[ic(i, j - 1, k)]) / dy;
            if (k >= 1)
                for (int64_t j = 0; j < ny; ++j)
                    for (int64_t i = 0; i < nx; ++i)
                        w[iw(i, j, k)] = ws[iw(i, j, k)] - scale * (p[ic(i, j, k)] - p[ic(i, j, k - 1)]) / dz;
        }
        return FLURSYS_OK;
    }

    // max_divergence (:504-517)
    double max_divergence() const override {
        double m = 0.0;
        for (int64_t k = 0; k < nz; ++k)
            for (int64_t j = 0; j < ny; ++j)
                for (int64_t i = 0; i < nx; ++i) {
                    double d = (u[iu(i + 1, j, k)] - u[iu(i, j, k)]) / dx +
                               (v[iv(i, j + 1, k)] - v[iv(i, j, k)]) / dy +
                               (w[iw(i, j, k + 1)] - w[iw(i, j, k)]) / dz;
                    m = std::max(m, std::fabs(d));
                }
        return m;
    }
    // max_speed (:519-532)
    double max_speed() const override {
        double m = 0.0;
        for (int64_t k = 0; k < nz; ++k)
            for (int64_t j = 0; j < ny; ++j)
                for (int64_t i = 0; i < nx; ++i) {
                    double a = 0.5 * (u[iu(i, j, k)] + u[iu(i + 1, j, k)]);
                    double b = 0.5 * (v[iv(i, j, k)] + v[iv(i, j + 1, k)]);
                    double c = 0.5 * (w[iw(i, j, k)] + w[iw(i, j, k + 1)]);
                    m = std::max(m, std::sqrt(a * a + b * b + c * c));
                }
        return m;
    }

    // advance_one_step (:164-172)
    int32_t advance(FlursysStepReport *rep) override {
        int32_t st = predict(dt);
        if (st) return st;
        rhs_phase(dt);
        double res = 0.0;
        int64_t its = 0;
        st = pressure(&res, &its);
        if (st) return st;
        correct(dt);
        step += 1;
        time = step * dt;
        // ensure_finite (:534-554)
        const char *names[4] = {"pressure", "u", "v", "w"};
        std::vector<double> *fs[4] = {&p, &u, &v, &w};
        for (int f = 0; f < 4; ++f) {
            size_t bad = 0;
            if (!all_finite(*fs[f], &bad)) {
                char buf[256];
                const double bv = (*fs[f])[bad];
                std::snprintf(buf, sizeof buf, "Non-finite 3D %s value at flat index %zu: %s",
                              names[f], bad, std::isnan(bv) ? "NaN" : (bv > 0 ? "inf" : "-inf"));
                err = buf;
                return FLURSYS_ERR_NON_FINITE;
            }
        }
        if (rep) {
            std::memset(rep, 0, sizeof *rep);
            rep->iteration = step;
            rep->time = time;
            rep->time_step = dt;
            rep->continuity_residual = max_divergence();
            rep->pressure_residual = res;
            rep->pressure_iterations = its;
            rep->max_speed = max_speed();
            rep->pressure_initial_residual = last_initial;
            rep->pressure_status = last_linear_status;
        }
        return FLURSYS_OK;
    }

    std::vector<double> *field(int32_t id) override {
        switch (id) {
            case FLURSYS_FIELD_U: return &u;
            case FLURSYS_FIELD_V: return &v;
            case FLURSYS_FIELD_W: return &w;
            case FLURSYS_FIELD_PRESSURE: return &p;
            case FLURSYS_FIELD_RHS: return &rhs;
            case FLURSYS_FIELD_U_STAR: return &us;
            case FLURSYS_FIELD_V_STAR: return &vs;
            case FLURSYS_FIELD_W_STAR: return &ws;
            default: return nullptr;
        }
    }
};

// ---------------------------------------------------------------------------
// 2D: IncompressibleSolver (incompressible.rs), without thermal physics.
// ---------------------------------------------------------------------------
struct Solver2D;

struct Operator2D final : StructuredOperator {
    const Solver2D *s;
    explicit Operator2D(const Solver2D *s_) : s(s_) {}
    bool identity_row(int64_t k) const override;
    double diagonal(int64_t k) const override;
    void apply(const std::vector<double> &x, std::vector<double> &y) const override;
    bool needs_projection() const override;
    void project(std::vector<double> &v) const override;
};

struct Solver2D final : OracleSolver {
    int64_t nx, ny;
    double dx, dy, length, height, rho, nu;
    CaseModel cm;
    std::vector<uint8_t> solid;
    std::vector<double> p, rhs, u, v, us, vs, uc, vc, speed, vort;
    std::vector<double> temp;  // cell temperature (empty when the energy model is off)
    bool thermal = false, boussinesq = false;
    double current_dt;

    size_t iu(int64_t i, int64_t j) const { return i + (nx + 1) * j; }
    size_t iv(int64_t i, int64_t j) const { return i + nx * j; }
    size_t ic(int64_t i, int64_t j) const { return i + nx * j; }
    bool sol(int64_t i, int64_t j) const { return solid[ic(i, j)] != 0; }

    explicit Solver2D(const FlursysCudaConfig &c) {
        cfg = c;
        nx = c.nx; ny = c.ny;
        length = c.case_params.length;
        height = c.case_params.height;
        dx = length / nx;
        dy = height / ny;
        rho = c.case_params.density;
        nu = c.case_params.kinematic_viscosity;
        cm.c = c.case_params;
        std::memcpy(cm.ov, c.overrides, sizeof cm.ov);
        solid.assign(nx * ny, 0);
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i)
                solid[ic(i, j)] = cm.is_solid((i + 0.5) * dx, (j + 0.5) * dy) ? 1 : 0;
        current_dt = c.dt;
        p.assign(nx * ny, 0.0);
        rhs = p; uc = p; vc = p; speed = p; vort = p;
        u.assign((nx + 1) * ny, 0.0);
        v.assign(nx * (ny + 1), 0.0);
        us = u; vs = v;
        thermal = c.physics.energy_model == FLURSYS_ENERGY_CONSTANT_PROPERTIES;
        boussinesq = c.physics.buoyancy == FLURSYS_BUOYANCY_BOUSSINESQ;
        if (thermal) temp.assign(nx * ny, c.physics.initial_temperature);  // :349-350
        initialize_velocity();
        compute_cell_fields();
    }

    // u_face_open / v_face_open (:2046-2064)
    bool u_open(int64_t i, int64_t j) const {
        if (i == 0) return !sol(0, j);
        if (i == nx) return !sol(nx - 1, j);
        return !sol(i - 1, j) && !sol(i, j);
    }
    bool v_open(int64_t i, int64_t j) const {
        if (j == 0) return !sol(i, 0);
        if (j == ny) return !sol(i, ny - 1);
        return !sol(i, j - 1) && !sol(i, j);
    }
    // pressure_outlet_cell (:2066-2080)
    bool outlet_cell(int64_t i, int64_t j) const {
        return i + 1 == nx && !sol(i, j) && cm.kind(FLURSYS_SIDE_RIGHT) == BK_OUTLET;
    }
    double outlet_pressure() const {
        double pr = 0.0;
        return cm.kind(FLURSYS_SIDE_RIGHT, &pr) == BK_OUTLET ? pr : 0.0;
    }
    bool reference_required() const { return cm.kind(FLURSYS_SIDE_RIGHT) != BK_OUTLET; }

    // tangential_ghost_u / tangential_ghost_v (:2159-2199)
    double ghost_u(int side, double center, double x) const {
        if (cm.kind(side) == BK_VELOCITY) {
            double y = side == FLURSYS_SIDE_BOTTOM ? 0.0 : height;
            double wu, wv;
            cm.velocity(side, x, y, &wu, &wv);
            return 2.0 * wu - center;
        }
        return center;
    }
    double ghost_v(int side, double center, double y) const {
        if (cm.kind(side) == BK_VELOCITY) {
            double x = side == FLURSYS_SIDE_LEFT ? 0.0 : length;
            double wu, wv;
            cm.velocity(side, x, y, &wu, &wv);
            return 2.0 * wv - center;
        }
        return center;
    }
    // MomentumStencil::u_neighbor / v_neighbor (:2089-2157)
    double u_nb(const std::vector<double> &uu, int64_t i, int64_t j, int di, int dj, double c) const {
        int64_t ii = i + di, jj = j + dj;
        if (ii >= 0 && ii <= nx && jj >= 0 && jj < ny) return u_open(ii, jj) ? uu[iu(ii, jj)] : -c;
        if (jj < 0) return ghost_u(FLURSYS_SIDE_BOTTOM, c, i * dx);
        if (jj >= ny) return ghost_u(FLURSYS_SIDE_TOP, c, i * dx);
        return c;
    }
    double v_nb(const std::vector<double> &vv, int64_t i, int64_t j, int di, int dj, double c) const {
        int64_t ii = i + di, jj = j + dj;
        if (ii >= 0 && ii < nx && jj >= 0 && jj <= ny) return v_open(ii, jj) ? vv[iv(ii, jj)] : -c;
        if (ii < 0) return ghost_v(FLURSYS_SIDE_LEFT, c, j * dy);
        if (ii >= nx) return ghost_v(FLURSYS_SIDE_RIGHT, c, j * dy);
        return c;
    }
    // transported (:2201-2212)
    double transported(double fv, double left, double right) const {
        if (cfg.convection == FLURSYS_CONVECTION_UPWIND) return fv >= 0.0 ? left : right;
        return 0.5 * (left + right);
    }

    // apply_velocity_boundaries (:1981-2044)
    void apply_boundaries(std::vector<double> &uu, std::vector<double> &vv) const {
        double bu, bv;
        for (int64_t j = 0; j < ny; ++j) {
            double y = (j + 0.5) * dy;
            switch (cm.kind(FLURSYS_SIDE_LEFT)) {
                case BK_VELOCITY: cm.velocity(FLURSYS_SIDE_LEFT, 0.0, y, &bu, &bv); uu[iu(0, j)] = bu; break;
                case BK_SYMMETRY: uu[iu(0, j)] = 0.0; break;
                case BK_OUTLET: uu[iu(0, j)] = uu[iu(1, j)]; break;
            }
            switch (cm.kind(FLURSYS_SIDE_RIGHT)) {
                case BK_VELOCITY: cm.velocity(FLURSYS_SIDE_RIGHT, length, y, &bu, &bv); uu[iu(nx, j)] = bu; break;
                case BK_SYMMETRY: uu[iu(nx, j)] = 0.0; break;
                case BK_OUTLET: uu[iu(nx, j)] = uu[iu(nx - 1, j)]; break;
            }
        }
        for (int64_t i = 0; i < nx; ++i) {
            double x = (i + 0.5) * dx;
            switch (cm.kind(FLURSYS_SIDE_BOTTOM)) {
                case BK_VELOCITY: cm.velocity(FLURSYS_SIDE_BOTTOM, x, 0.0, &bu, &bv); vv[iv(i, 0)] = bv; break;
                case BK_SYMMETRY: vv[iv(i, 0)] = 0.0; break;
                case BK_OUTLET: vv[iv(i, 0)] = vv[iv(i, 1)]; break;
            }
            switch (cm.kind(FLURSYS_SIDE_TOP)) {
                case BK_VELOCITY: cm.velocity(FLURSYS_SIDE_TOP, x, height, &bu, &bv); vv[iv(i, ny)] = bv; break;
                case BK_SYMMETRY: vv[iv(i, ny)] = 0.0; break;
                case BK_OUTLET: vv[iv(i, ny)] = vv[iv(i, ny - 1)]; break;
            }
        }
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 1; i < nx; ++i)
                if (!u_open(i, j)) uu[iu(i, j)] = 0.0;
        for (int64_t j = 1; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i)
                if (!v_open(i, j)) vv[iv(i, j)] = 0.0;
    }

    // initialize_velocity (:588-620)
    void initialize_velocity() {
        double a, b;
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i <= nx; ++i) {
                cm.initial_velocity(i * dx, (j + 0.5) * dy, &a, &b);
                u[iu(i, j)] = u_open(i, j) ? a : 0.0;
            }
        for (int64_t j = 0; j <= ny; ++j)
            for (int64_t i = 0; i < nx; ++i) {
                cm.initial_velocity((i + 0.5) * dx, j * dy, &a, &b);
                v[iv(i, j)] = v_open(i, j) ? b : 0.0;
            }
        apply_boundaries(u, v);
    }

    bool simple() const { return cfg.coupling == FLURSYS_COUPLING_SIMPLE; }

    // predict_momentum (:748-922), with the Boussinesq body force
    // g * beta * (face temperature - T_ref) (:831-846, :896-911) when the
    // buoyancy model is on and a temperature field exists (0.0 otherwise).
    int32_t predict(double step_dt) override {
        std::fill(us.begin(), us.end(), 0.0);
        std::fill(vs.begin(), vs.end(), 0.0);
        const bool with_p = simple();
        const double relax = with_p ? cfg.velocity_relaxation : 1.0;
        const bool buoy = boussinesq && thermal;
        const double tref = boussinesq ? cfg.physics.reference_temperature : 0.0;
        const double gbx = cfg.physics.gravity_x * cfg.physics.thermal_expansion;
        const double gby = cfg.physics.gravity_y * cfg.physics.thermal_expansion;
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 1; i < nx; ++i) {
                if (!u_open(i, j)) continue;
                double up = u[iu(i, j)];
                double ue_nb = u_nb(u, i, j, 1, 0, up), uw_nb = u_nb(u, i, j, -1, 0, up);
                double un_nb = u_nb(u, i, j, 0, 1, up), us_nb = u_nb(u, i, j, 0, -1, up);
                double ue = 0.5 * (up + ue_nb), uw = 0.5 * (uw_nb + up);
                double vn = 0.5 * (v[iv(i - 1, j + 1)] + v[iv(i, j + 1)]);
                double vsf = 0.5 * (v[iv(i - 1, j)] + v[iv(i, j)]);
                double pe = transported(ue, up, ue_nb), pw = transported(uw, uw_nb, up);
                double pn = transported(vn, up, un_nb), ps = transported(vsf, us_nb, up);
                double conv = (ue * pe - uw * pw) / dx + (vn * pn - vsf * ps) / dy;
                double diff = (ue_nb - 2.0 * up + uw_nb) / (dx * dx) + (un_nb - 2.0 * up + us_nb) / (dy * dy);
                double pg = with_p ? (p[ic(i, j)] - p[ic(i - 1, j)]) / dx : 0.0;
                double bx = buoy ? gbx * (0.5 * (temp[ic(i - 1, j)] + temp[ic(i, j)]) - tref) : 0.0;
                us[iu(i, j)] = up + relax * step_dt * (-conv + nu * diff - pg / rho + bx);
            }
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
        for (int64_t j = 1; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i) {
                if (!v_open(i, j)) continue;
                double vp = v[iv(i, j)];
                double ve_nb = v_nb(v, i, j, 1, 0, vp), vw_nb = v_nb(v, i, j, -1, 0, vp);
                double vn_nb = v_nb(v, i, j, 0, 1, vp), vs_nb = v_nb(v, i, j, 0, -1, vp);
                double ue = 0.5 * (u[iu(i + 1, j - 1)] + u[iu(i + 1, j)]);
                double uw = 0.5 * (u[iu(i, j - 1)] + u[iu(i, j)]);
                double vn = 0.5 * (vp + vn_nb), vsf = 0.5 * (vs_nb + vp);
                double pe = transported(ue, vp, ve_nb), pw = transported(uw, vw_nb, vp);
                double pn = transported(vn, vp, vn_nb), ps = transported(vsf, vs_nb, vp);
                double conv = (ue * pe - uw * pw) / dx + (vn * pn - vsf * ps) / dy;
                double diff = (ve_nb - 2.0 * vp + vw_nb) / (dx * dx) + (vn_nb - 2.0 * vp + vs_nb) / (dy * dy);
                double pg = with_p ? (p[ic(i, j)] - p[ic(i, j - 1)]) / dy : 0.0;
                double by = buoy ? gby * (0.5 * (temp[ic(i, j - 1)] + temp[ic(i, j)]) - tref) : 0.0;
                vs[iv(i, j)] = vp + relax * step_dt * (-conv + nu * diff - pg / rho + by);
            }
        return FLURSYS_OK;
    }

    // build_pressure_rhs (:924-970)
    int32_t rhs_phase(double step_dt) override {
        const double scale = simple() ? cfg.velocity_relaxation : 1.0;
        const double rho_over_dt = rho / (scale * step_dt);
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i) {
                if (sol(i, j) || outlet_cell(i, j)) {
                    rhs[ic(i, j)] = 0.0;
                    continue;
                }
                double div = (us[iu(i + 1, j)] - us[iu(i, j)]) / dx + (vs[iv(i, j + 1)] - vs[iv(i, j)]) / dy;
                rhs[ic(i, j)] = rho_over_dt * div;
            }
        return FLURSYS_OK;
    }

    // pressure_residual (:1532-1567)
    double pressure_residual() const override {
        const double idx2 = 1.0 / (dx * dx), idy2 = 1.0 / (dy * dy);
        double m = 0.0;
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i) {
                if (sol(i, j) || outlet_cell(i, j)) continue;
                double p0 = p[ic(i, j)];
                double pe = (i + 1 < nx && !sol(i + 1, j)) ? p[ic(i + 1, j)] : p0;
                double pw = (i > 0 && !sol(i - 1, j)) ? p[ic(i - 1, j)] : p0;
                double pn = (j + 1 < ny && !sol(i, j + 1)) ? p[ic(i, j + 1)] : p0;
                double ps = (j > 0 && !sol(i, j - 1)) ? p[ic(i, j - 1)] : p0;
                double lap = (pe - 2.0 * p0 + pw) * idx2 + (pn - 2.0 * p0 + ps) * idy2;
                m = std::max(m, std::fabs(lap - rhs[ic(i, j)]));
            }
        return m;
    }

    // solve_pressure_sor (:979-1046)
    int32_t pressure_sor(double *res_out, int64_t *its_out) {
        const double idx2 = 1.0 / (dx * dx), idy2 = 1.0 / (dy * dy);
        const double omega = cfg.pressure_omega;
        double residual = INFINITY;
        int64_t its = 0;
        for (int64_t it = 0; it < cfg.pressure_max_iters; ++it) {
            its = it + 1;
            for (int64_t j = 0; j < ny; ++j)
                for (int64_t i = 0; i < nx; ++i) {
                    if (sol(i, j)) { p[ic(i, j)] = 0.0; continue; }
                    if (outlet_cell(i, j)) { p[ic(i, j)] = outlet_pressure(); continue; }
                    double ap = 0.0, s = 0.0;
                    if (i + 1 < nx && !sol(i + 1, j)) { ap += idx2; s += idx2 * p[ic(i + 1, j)]; }
                    if (i > 0 && !sol(i - 1, j)) { ap += idx2; s += idx2 * p[ic(i - 1, j)]; }
                    if (j + 1 < ny && !sol(i, j + 1)) { ap += idy2; s += idy2 * p[ic(i, j + 1)]; }
                    if (j > 0 && !sol(i, j - 1)) { ap += idy2; s += idy2 * p[ic(i, j - 1)]; }
                    if (ap > 0.0) {
                        double cand = (s - rhs[ic(i, j)]) / ap;
                        double old = p[ic(i, j)];
                        p[ic(i, j)] = old + omega * (cand - old);
                    }
                }
            if (reference_required()) {
                int64_t ref = -1;  // find_reference_cell (:1614-1623)
                for (int64_t k = 0; k < nx * ny && ref < 0; ++k)
                    if (!solid[k]) ref = k;
                if (ref >= 0) {
                    double pr = p[ref];
                    for (int64_t k = 0; k < nx * ny; ++k)
                        if (!solid[k]) p[k] -= pr;
                }
            }
            residual = pressure_residual();
            if (!std::isfinite(residual)) {
                err = "Pressure solver produced a non-finite residual";
                return FLURSYS_ERR_NON_FINITE;
            }
            if (residual < cfg.pressure_tolerance) break;
        }
        *res_out = residual;
        *its_out = its;
        return FLURSYS_OK;
    }

    double last_initial = 0.0;
    int32_t last_linear_status = FLURSYS_LINEAR_CONVERGED;

    // solve_pressure_pcg (:1048-1214)
    int32_t pressure(double *res_out, int64_t *its_out) override {
        if (cfg.pressure_solver == FLURSYS_PRESSURE_SOR) return pressure_sor(res_out, its_out);
        const int64_t n = nx * ny;
        std::vector<double> x(p), b(n);
        const double op_ = outlet_pressure();
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i) {
                int64_t k = ic(i, j);
                if (sol(i, j) || outlet_cell(i, j)) {
                    double val = outlet_cell(i, j) ? op_ : 0.0;
                    x[k] = val;
                    b[k] = val;
                } else {
                    b[k] = -rhs[k];
                }
            }
        Operator2D op(this);
        StopRule stop;
        stop.rule = cfg.stop_rule == FLURSYS_STOP_REL_L2 ? FLURSYS_STOP_REL_L2 : FLURSYS_STOP_ABS_INF;
        stop.tol = cfg.pressure_tolerance;
        stop.atol = cfg.pressure_atol;
        stop.rtol = cfg.pressure_rtol;
        PcgResult r = pcg_core(op, b, x, stop, cfg.pressure_max_iters);
        if (r.status != FLURSYS_OK) {
            err = r.error;
            return r.status;
        }
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i) {
                int64_t k = ic(i, j);
                p[k] = sol(i, j) ? 0.0 : (outlet_cell(i, j) ? op_ : x[k]);
            }
        last_initial = r.initial;
        last_linear_status = r.linear_status;
        *res_out = r.residual;
        *its_out = r.iterations;
        return FLURSYS_OK;
    }

    // correct_velocity (:1322-1379)
    int32_t correct(double step_dt) override {
        const double scale = simple() ? cfg.velocity_relaxation : 1.0;
        const double dt_over_rho = scale * step_dt / rho;
        u = us;
        v = vs;
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 1; i < nx; ++i)
                u[iu(i, j)] = u_open(i, j) ? us[iu(i, j)] - dt_over_rho * ((p[ic(i, j)] - p[ic(i - 1, j)]) / dx) : 0.0;
        for (int64_t j = 1; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i)
                v[iv(i, j)] = v_open(i, j) ? vs[iv(i, j)] - dt_over_rho * ((p[ic(i, j)] - p[ic(i, j - 1)]) / dy) : 0.0;
        return FLURSYS_OK;
    }

    // derivative_x_slice / derivative_y_slice (:2227-2285)
    double ddx_cell(const std::vector<double> &f, int64_t i, int64_t j) const {
        double c = f[ic(i, j)];
        bool e_ok = i + 1 < nx && !sol(i + 1, j), w_ok = i > 0 && !sol(i - 1, j);
        double e = e_ok ? f[ic(i + 1, j)] : c, w = w_ok ? f[ic(i - 1, j)] : c;
        if (e_ok && w_ok) return (e - w) / (2.0 * dx);
        if (e_ok) return (e - c) / dx;
        if (w_ok) return (c - w) / dx;
        return 0.0;
    }
    double ddy_cell(const std::vector<double> &f, int64_t i, int64_t j) const {
        double c = f[ic(i, j)];
        bool n_ok = j + 1 < ny && !sol(i, j + 1), s_ok = j > 0 && !sol(i, j - 1);
        double n = n_ok ? f[ic(i, j + 1)] : c, s = s_ok ? f[ic(i, j - 1)] : c;
        if (n_ok && s_ok) return (n - s) / (2.0 * dy);
        if (n_ok) return (n - c) / dy;
        if (s_ok) return (c - s) / dy;
        return 0.0;
    }
    // compute_cell_fields (:1381-1439)
    void compute_cell_fields() {
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i) {
                int64_t k = ic(i, j);
                if (sol(i, j)) { uc[k] = vc[k] = speed[k] = 0.0; continue; }
                double a = 0.5 * (u[iu(i, j)] + u[iu(i + 1, j)]);
                double b = 0.5 * (v[iv(i, j)] + v[iv(i, j + 1)]);
                uc[k] = a;
                vc[k] = b;
                speed[k] = std::sqrt(a * a + b * b);
            }
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i)
                vort[ic(i, j)] = sol(i, j) ? 0.0 : ddx_cell(vc, i, j) - ddy_cell(uc, i, j);
    }
    // max_divergence (:1569-1582)
    double max_divergence() const override {
        double m = 0.0;
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i) {
                if (sol(i, j)) continue;
                double d = (u[iu(i + 1, j)] - u[iu(i, j)]) / dx + (v[iv(i, j + 1)] - v[iv(i, j)]) / dy;
                m = std::max(m, std::fabs(d));
            }
        return m;
    }
    double max_speed() const override { return field_max_abs(speed); }

    // cylinder_force_coefficients (:1634-1676)
    void forces(double *cd, double *cl) const {
        *cd = *cl = 0.0;
        if (cm.c.kind != FLURSYS_CASE_CYLINDER) return;
        double mu = cm.c.cylinder_mu, fx = 0.0, fy = 0.0;
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i) {
                if (sol(i, j)) continue;
                double pp = p[ic(i, j)], a = uc[ic(i, j)], b = vc[ic(i, j)];
                if (i + 1 < nx && sol(i + 1, j)) { fx += pp * dy; fy += mu * b / (0.5 * dx) * dy; }
                if (i > 0 && sol(i - 1, j)) { fx -= pp * dy; fy += mu * b / (0.5 * dx) * dy; }
                if (j + 1 < ny && sol(i, j + 1)) { fy += pp * dx; fx += mu * a / (0.5 * dy) * dx; }
                if (j > 0 && sol(i, j - 1)) { fy -= pp * dx; fx += mu * a / (0.5 * dy) * dx; }
            }
        double q = 0.5 * rho * cm.c.reference_velocity * cm.c.reference_velocity * cm.c.cylinder_diameter;
        if (q > 0.0) { *cd = fx / q; *cl = fy / q; }
    }

    // temperature_neighbor (:1495-1530): solid neighbours and adiabatic
    // walls mirror the centre, a fixed-temperature wall is 2 T_w - centre.
    double temp_nb(const std::vector<double> &t, int64_t i, int64_t j, int di, int dj, double center) const {
        const int64_t ni = i + di, nj = j + dj;
        if (ni >= 0 && ni < nx && nj >= 0 && nj < ny) return sol(ni, nj) ? center : t[ic(ni, nj)];
        const int side = ni < 0 ? FLURSYS_SIDE_LEFT
                                : (ni >= nx ? FLURSYS_SIDE_RIGHT : (nj < 0 ? FLURSYS_SIDE_BOTTOM : FLURSYS_SIDE_TOP));
        const FlursysThermalBoundary &b = cfg.physics.thermal[side];
        return b.kind == FLURSYS_THERMAL_FIXED_TEMPERATURE ? 2.0 * b.temperature - center : center;
    }
    // advance_temperature (:1441-1493): explicit conservative upwind update
    // on the new face velocities, after the runtime thermal CFL check.
    int32_t advance_temperature(double step_dt) {
        if (!thermal) return FLURSYS_OK;
        const double cfl = step_dt * (field_max_abs(uc) / dx + field_max_abs(vc) / dy);
        if (cfl > 1.0) {
            err = "explicit thermal advection is unstable at step " + std::to_string((long long)step) +
                  ": CFL=" + rust_sci(cfl, 3) + " exceeds 1";
            return FLURSYS_ERR_INVALID_CONFIG;
        }
        const std::vector<double> old = temp;
        const double alpha = cfg.physics.thermal_diffusivity, source = cfg.physics.source_temperature_rate;
        auto upw = [](double fv, double pos, double neg) { return fv >= 0.0 ? pos : neg; };
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i) {
                const int64_t k = ic(i, j);
                if (sol(i, j)) { temp[k] = old[k]; continue; }
                const double c = old[k];
                const double e = temp_nb(old, i, j, 1, 0, c), w = temp_nb(old, i, j, -1, 0, c);
                const double n = temp_nb(old, i, j, 0, 1, c), so = temp_nb(old, i, j, 0, -1, c);
                const double ue = u[iu(i + 1, j)], uw = u[iu(i, j)], vn = v[iv(i, j + 1)], vsf = v[iv(i, j)];
                const double fe = ue * upw(ue, c, e), fw = uw * upw(uw, w, c);
                const double fn = vn * upw(vn, c, n), fs = vsf * upw(vsf, so, c);
                const double conv = (fe - fw) / dx + (fn - fs) / dy;
                const double diff = (e - 2.0 * c + w) / (dx * dx) + (n - 2.0 * c + so) / (dy * dy);
                temp[k] = c + step_dt * (-conv + alpha * diff + source);
            }
        return FLURSYS_OK;
    }

    // reached_end_time (:557-561)
    bool reached_end_time() const {
        double tol = 2.220446049250313e-16 * std::max(std::fabs(cfg.t_end), 1.0) * 16.0;
        return cfg.coupling == FLURSYS_COUPLING_PROJECTION && time >= cfg.t_end - tol;
    }

    // advance_one_step (:622-746) + advance() (:523-555)
    int32_t advance(FlursysStepReport *rep) override {
        if (reached_end_time()) {
            err = "projection simulation has already reached t_end";
            return FLURSYS_ERR_REACHED_END_TIME;
        }
        double step_dt = cfg.dt;
        if (cfg.adaptive) {
            int32_t st = adaptive_dt(current_dt, field_max_abs(u), field_max_abs(v), dx, dy, nu,
                                     thermal ? cfg.physics.thermal_diffusivity : -1.0,
                                     cfg.min_dt, cfg.max_dt, cfg.target_cfl, cfg.target_diffusion_number,
                                     cfg.max_growth_factor, &step_dt, &err);
            if (st) return st;
        }
        if (cfg.coupling == FLURSYS_COUPLING_PROJECTION) {
            double remaining = cfg.t_end - time;
            step_dt = std::min(step_dt, remaining);
            if (step_dt <= 0.0) {
                err = "projection simulation has already reached t_end";
                return FLURSYS_ERR_REACHED_END_TIME;
            }
        }
        if (cfg.adaptive) current_dt = step_dt;
        std::vector<double> old_u(u), old_v(v);
        const bool smp = simple();
        predict(step_dt);
        apply_boundaries(us, vs);
        std::vector<double> old_p;
        if (smp) {
            old_p = p;
            std::fill(p.begin(), p.end(), 0.0);
        }
        rhs_phase(step_dt);
        double res = 0.0;
        int64_t its = 0;
        int32_t st = pressure(&res, &its);
        if (st) return st;
        correct(step_dt);
        if (smp)
            for (size_t k = 0; k < p.size(); ++k) p[k] = old_p[k] + cfg.pressure_relaxation * p[k];
        apply_boundaries(u, v);
        step += 1;
        if (cfg.coupling == FLURSYS_COUPLING_PROJECTION) time += step_dt;
        else time = step * cfg.dt;
        compute_cell_fields();
        if (int32_t tst = advance_temperature(step_dt)) return tst;
        // ensure_finite (:1707-1742)
        const char *names[5] = {"pressure", "u", "v", "speed", "temperature"};
        std::vector<double> *fs[5] = {&p, &u, &v, &speed, &temp};
        for (int f = 0; f < 5; ++f) {
            size_t bad = 0;
            if (!all_finite(*fs[f], &bad)) {
                char buf[256];
                const double bv = (*fs[f])[bad];
                std::snprintf(buf, sizeof buf, "Non-finite %s value at flat index %zu: %s (step %lld)",
                              names[f], bad, std::isnan(bv) ? "NaN" : (bv > 0 ? "inf" : "-inf"), (long long)step);
                err = buf;
                return FLURSYS_ERR_NON_FINITE;
            }
        }
        double mu_ = field_max_abs(u), mv_ = field_max_abs(v);
        double vel_change = 0.0;
        for (size_t k = 0; k < u.size(); ++k) vel_change = std::max(vel_change, std::fabs(u[k] - old_u[k]));
        double vch = 0.0;
        for (size_t k = 0; k < v.size(); ++k) vch = std::max(vch, std::fabs(v[k] - old_v[k]));
        vel_change = std::max(vel_change, vch);
        if (rep) {
            std::memset(rep, 0, sizeof *rep);
            rep->iteration = step;
            rep->time = time;
            rep->time_step = step_dt;
            rep->continuity_residual = max_divergence();
            rep->pressure_residual = res;
            rep->pressure_iterations = its;
            rep->momentum_residual = vel_change;
            rep->max_speed = max_speed();
            rep->momentum_cfl = step_dt * (mu_ / dx + mv_ / dy);
            rep->viscous_diffusion_number = nu * step_dt * (1.0 / (dx * dx) + 1.0 / (dy * dy));
            forces(&rep->drag_coefficient, &rep->lift_coefficient);
            rep->converged = cm.c.kind != FLURSYS_CASE_CYLINDER && step >= cfg.minimum_steps &&
                             vel_change < cfg.steady_tolerance &&
                             rep->continuity_residual < 10.0 * cfg.pressure_tolerance;
            rep->reached_end_time = reached_end_time();
            rep->pressure_initial_residual = last_initial;
            rep->pressure_status = last_linear_status;
        }
        return FLURSYS_OK;
    }

    std::vector<double> *field(int32_t id) override {
        switch (id) {
            case FLURSYS_FIELD_U: return &u;
            case FLURSYS_FIELD_V: return &v;
            case FLURSYS_FIELD_PRESSURE: return &p;
            case FLURSYS_FIELD_RHS: return &rhs;
            case FLURSYS_FIELD_U_STAR: return &us;
            case FLURSYS_FIELD_V_STAR: return &vs;
            case FLURSYS_FIELD_SPEED: return &speed;
            case FLURSYS_FIELD_VORTICITY: return &vort;
            case FLURSYS_FIELD_U_CELL: return &uc;
            case FLURSYS_FIELD_V_CELL: return &vc;
            case FLURSYS_FIELD_TEMPERATURE: return thermal ? &temp : nullptr;
            default: return nullptr;
        }
    }
};

bool Operator2D::identity_row(int64_t k) const {
    int64_t i = k % s->nx, j = k / s->nx;
    return s->sol(i, j) || s->outlet_cell(i, j);
}
double Operator2D::diagonal(int64_t k) const {
    int64_t i = k % s->nx, j = k / s->nx;
    const double idx2 = 1.0 / (s->dx * s->dx), idy2 = 1.0 / (s->dy * s->dy);
    if (identity_row(k)) return 0.0;
    double dg = 0.0;
    if (i + 1 < s->nx && !s->sol(i + 1, j)) dg += idx2;
    if (i > 0 && !s->sol(i - 1, j)) dg += idx2;
    if (j + 1 < s->ny && !s->sol(i, j + 1)) dg += idy2;
    if (j > 0 && !s->sol(i, j - 1)) dg += idy2;
    return dg;
}
// apply_pressure_operator (:1216-1255)
void Operator2D::apply(const std::vector<double> &x, std::vector<double> &y) const {
    const int64_t nx = s->nx, ny = s->ny;
    const double idx2 = 1.0 / (s->dx * s->dx), idy2 = 1.0 / (s->dy * s->dy);
#pragma omp parallel for num_threads(g_threads) schedule(static) if (g_threads > 1)
    for (int64_t j = 0; j < ny; ++j)
        for (int64_t i = 0; i < nx; ++i) {
            int64_t k = i + nx * j;
            if (s->sol(i, j) || s->outlet_cell(i, j)) { y[k] = x[k]; continue; }
            double dg = 0.0, nb = 0.0;
            if (i + 1 < nx && !s->sol(i + 1, j)) { dg += idx2; nb += idx2 * x[k + 1]; }
            if (i > 0 && !s->sol(i - 1, j)) { dg += idx2; nb += idx2 * x[k - 1]; }
            if (j + 1 < ny && !s->sol(i, j + 1)) { dg += idy2; nb += idy2 * x[k + nx]; }
            if (j > 0 && !s->sol(i, j - 1)) { dg += idy2; nb += idy2 * x[k - nx]; }
            y[k] = dg * x[k] - nb;
        }
}
bool Operator2D::needs_projection() const { return s->reference_required(); }
// project_zero_mean (:2338-2377) over fluid, non-Dirichlet cells.
void Operator2D::project(std::vector<double> &vals) const {
    const int64_t nx = s->nx, ny = s->ny;
    double sum = 0.0;
    int64_t count = 0;
    for (int64_t j = 0; j < ny; ++j) {
        double row = 0.0;
        int64_t rc = 0;
        for (int64_t i = 0; i < nx; ++i)
            if (!s->sol(i, j) && !s->outlet_cell(i, j)) { row += vals[i + nx * j]; rc += 1; }
        sum += row;
        count += rc;
    }
    if (count == 0) return;
    double mean = sum / (double)count;
    for (int64_t j = 0; j < ny; ++j)
        for (int64_t i = 0; i < nx; ++i)
            if (!s->sol(i, j) && !s->outlet_cell(i, j)) vals[i + nx * j] -= mean;
}

// Pure-Neumann 2D operator without solids for orc_stencil_pcg (the cavity
// operator of apply_pressure_operator with zero-mean projections).
struct Neumann2DOperator final : StructuredOperator {
    int64_t nx, ny;
    double idx2, idy2;
    Neumann2DOperator(int64_t nx_, int64_t ny_, double dx, double dy)
        : nx(nx_), ny(ny_), idx2(1.0 / (dx * dx)), idy2(1.0 / (dy * dy)) {}
    bool identity_row(int64_t) const override { return false; }
    double diagonal(int64_t k) const override {
        int64_t i = k % nx, j = k / nx;
        double dg = 0.0;
        if (i + 1 < nx) dg += idx2;
        if (i > 0) dg += idx2;
        if (j + 1 < ny) dg += idy2;
        if (j > 0) dg += idy2;
        return dg;
    }
    void apply(const std::vector<double> &x, std::vector<double> &y) const override {
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i) {
                int64_t k = i + nx * j;
                double dg = 0.0, nb = 0.0;
                if (i + 1 < nx) { dg += idx2; nb += idx2 * x[k + 1]; }
                if (i > 0) { dg += idx2; nb += idx2 * x[k - 1]; }
                if (j + 1 < ny) { dg += idy2; nb += idy2 * x[k + nx]; }
                if (j > 0) { dg += idy2; nb += idy2 * x[k - nx]; }
                y[k] = dg * x[k] - nb;
            }
    }
    bool needs_projection() const override { return true; }
    void project(std::vector<double> &vals) const override {
        double sum = 0.0;
        for (int64_t j = 0; j < ny; ++j) {
            double row = 0.0;
            for (int64_t i = 0; i < nx; ++i) row += vals[i + nx * j];
            sum += row;
        }
        double mean = sum / (double)(nx * ny);
        for (auto &x : vals) x -= mean;
    }
};

// ---------------------------------------------------------------------------
// src/linear: CSR (csr.rs), Jacobi (preconditioner.rs), solvers (solver.rs).
// ---------------------------------------------------------------------------
struct Csr {
    int64_t nrows, ncols;
    const int64_t *ro;
    const int64_t *ci;
    const double *v;
};

// validate_csr (csr.rs:194-247)
int32_t validate_csr(int64_t nrows, int64_t ncols, int64_t nnz, const int64_t *ro, const int64_t *ci,
                     const double *v, std::string *msg) {
    if (!ro) { *msg = "row_offsets length must equal nrows + 1"; return FLURSYS_ERR_INVALID_CSR; }
    if (ro[0] != 0) { *msg = "first row offset must be zero"; return FLURSYS_ERR_INVALID_CSR; }
    if (ro[nrows] != nnz) { *msg = "last row offset must equal value count"; return FLURSYS_ERR_INVALID_CSR; }
    for (int64_t r = 0; r < nrows; ++r) {
        if (ro[r] > ro[r + 1]) { *msg = "row offsets must be monotonic"; return FLURSYS_ERR_INVALID_CSR; }
        for (int64_t e = ro[r] + 1; e < ro[r + 1]; ++e)
            if (ci[e - 1] >= ci[e]) { *msg = "row columns must be strictly ascending"; return FLURSYS_ERR_INVALID_CSR; }
    }
    for (int64_t e = 0; e < nnz; ++e)
        if (ci[e] < 0 || ci[e] >= ncols) {
            char buf[128];
            std::snprintf(buf, sizeof buf, "column %lld at entry %lld exceeds ncols", (long long)ci[e], (long long)e);
            *msg = buf;
            return FLURSYS_ERR_INVALID_CSR;
        }
    for (int64_t e = 0; e < nnz; ++e)
        if (!std::isfinite(v[e])) { *msg = "non-finite matrix value"; return FLURSYS_ERR_NON_FINITE; }
    return FLURSYS_OK;
}

// spmv_into (csr.rs:89-106)
int32_t spmv(const Csr &a, const double *x, double *y) {
    for (int64_t r = 0; r < a.nrows; ++r) {
        double s = 0.0;
        for (int64_t e = a.ro[r]; e < a.ro[r + 1]; ++e) s += a.v[e] * x[a.ci[e]];
        if (!std::isfinite(s)) return FLURSYS_ERR_NON_FINITE;
        y[r] = s;
    }
    return FLURSYS_OK;
}

// diagonal_entry (csr.rs:67-82) + JacobiPreconditioner::new (preconditioner.rs:10-30)
int32_t jacobi(const Csr &a, std::vector<double> &inv, int64_t *bad) {
    inv.assign(a.nrows, 0.0);
    for (int64_t r = 0; r < a.nrows; ++r) {
        const int64_t *b = a.ci + a.ro[r], *e = a.ci + a.ro[r + 1];
        const int64_t *f = std::lower_bound(b, e, r);
        if (f == e || *f != r) { *bad = r; return FLURSYS_ERR_MISSING_DIAGONAL; }
        double d = a.v[a.ro[r] + (f - b)];
        if (!std::isfinite(d)) { *bad = r; return FLURSYS_ERR_NON_FINITE; }
        if (d == 0.0) { *bad = r; return FLURSYS_ERR_ZERO_DIAGONAL; }
        double iv = 1.0 / d;
        if (!std::isfinite(iv)) { *bad = r; return FLURSYS_ERR_NON_FINITE; }
        inv[r] = iv;
    }
    return FLURSYS_OK;
}

double sdot(const double *a, const double *b, int64_t n) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

void fill_report(FlursysLinearSolveReport *rep, int32_t status, int64_t its, double initial, double fin) {
    if (!rep) return;
    rep->status = status;
    rep->reserved = 0;
    rep->iterations = its;
    rep->initial_residual = initial;
    rep->final_residual = fin;
    rep->relative_residual = initial == 0.0 ? 0.0 : fin / initial;
}

// validate_solve_inputs (solver.rs:258-300); dimensions are implied by n here.
int32_t validate_inputs(int64_t n, const double *rhs, const double *x, const FlursysLinearSolverOptions &o) {
    if (!std::isfinite(o.absolute_tolerance) || o.absolute_tolerance < 0.0 ||
        !std::isfinite(o.relative_tolerance) || o.relative_tolerance < 0.0)
        return FLURSYS_ERR_BREAKDOWN;
    for (int64_t i = 0; i < n; ++i)
        if (!std::isfinite(rhs[i])) return FLURSYS_ERR_NON_FINITE;
    for (int64_t i = 0; i < n; ++i)
        if (!std::isfinite(x[i])) return FLURSYS_ERR_NON_FINITE;
    return FLURSYS_OK;
}

// solve_cg (solver.rs:62-153)
int32_t solve_cg(const Csr &a, const double *rhs, double *x, const FlursysLinearSolverOptions &o,
                 const std::vector<double> *inv, FlursysLinearSolveReport *rep) {
    const int64_t n = a.nrows;
    int32_t st = validate_inputs(n, rhs, x, o);
    if (st) return st;
    std::vector<double> r(n), d(n), q(n), z(n);
    if ((st = spmv(a, x, r.data()))) return st;
    for (int64_t i = 0; i < n; ++i) {
        r[i] = rhs[i] - r[i];
        if (!std::isfinite(r[i])) return FLURSYS_ERR_NON_FINITE;
    }
    double initial = std::sqrt(sdot(r.data(), r.data(), n));
    if (!std::isfinite(initial)) return FLURSYS_ERR_NON_FINITE;
    double threshold = o.absolute_tolerance + o.relative_tolerance * initial;
    if (initial <= threshold) { fill_report(rep, FLURSYS_LINEAR_CONVERGED, 0, initial, initial); return FLURSYS_OK; }
    auto precond = [&]() -> int32_t {
        if (inv) {
            for (int64_t i = 0; i < n; ++i) {
                z[i] = r[i] * (*inv)[i];
                if (!std::isfinite(z[i])) return FLURSYS_ERR_NON_FINITE;
            }
        } else {
            z = r;
        }
        return FLURSYS_OK;
    };
    if ((st = precond())) return st;
    d = z;
    double rho = sdot(r.data(), z.data(), n);
    if (!std::isfinite(rho)) return FLURSYS_ERR_NON_FINITE;
    for (int64_t it = 1; it <= o.max_iterations; ++it) {
        if ((st = spmv(a, d.data(), q.data()))) return st;
        double den = sdot(d.data(), q.data(), n);
        if (!std::isfinite(den) || std::fabs(den) <= 1.0e-30) return FLURSYS_ERR_BREAKDOWN;
        double alpha = rho / den;
        if (!std::isfinite(alpha)) return FLURSYS_ERR_BREAKDOWN;
        for (int64_t i = 0; i < n; ++i) {
            x[i] += alpha * d[i];
            r[i] -= alpha * q[i];
        }
        double rn2 = sdot(r.data(), r.data(), n);
        if (!std::isfinite(rn2)) return FLURSYS_ERR_NON_FINITE;
        double rn = std::sqrt(rn2);
        if (rn <= threshold) { fill_report(rep, FLURSYS_LINEAR_CONVERGED, it, initial, rn); return FLURSYS_OK; }
        if ((st = precond())) return st;
        double rho_new = sdot(r.data(), z.data(), n);
        if (!std::isfinite(rho_new) || std::fabs(rho) <= 1.0e-30) return FLURSYS_ERR_BREAKDOWN;
        double beta = rho_new / rho;
        if (!std::isfinite(beta)) return FLURSYS_ERR_BREAKDOWN;
        for (int64_t i = 0; i < n; ++i) d[i] = z[i] + beta * d[i];
        rho = rho_new;
    }
    double fin = std::sqrt(sdot(r.data(), r.data(), n));
    fill_report(rep, FLURSYS_LINEAR_MAX_ITERATIONS, o.max_iterations, initial, fin);
    return FLURSYS_OK;
}

// bicgstab (solver.rs:155-256)
int32_t solve_bicgstab(const Csr &a, const double *rhs, double *x, const FlursysLinearSolverOptions &o,
                       FlursysLinearSolveReport *rep) {
    const int64_t n = a.nrows;
    int32_t st = validate_inputs(n, rhs, x, o);
    if (st) return st;
    std::vector<double> r(n), rh, p(n, 0.0), v(n, 0.0), s(n), t(n);
    if ((st = spmv(a, x, r.data()))) return st;
    for (int64_t i = 0; i < n; ++i) {
        r[i] = rhs[i] - r[i];
        if (!std::isfinite(r[i])) return FLURSYS_ERR_NON_FINITE;
    }
    rh = r;
    double initial = std::sqrt(sdot(r.data(), r.data(), n));
    if (!std::isfinite(initial)) return FLURSYS_ERR_NON_FINITE;
    double threshold = o.absolute_tolerance + o.relative_tolerance * initial;
    if (initial <= threshold) { fill_report(rep, FLURSYS_LINEAR_CONVERGED, 0, initial, initial); return FLURSYS_OK; }
    double rho_prev = 1.0, alpha = 1.0, omega = 1.0;
    for (int64_t it = 1; it <= o.max_iterations; ++it) {
        double rho = sdot(rh.data(), r.data(), n);
        if (!std::isfinite(rho) || std::fabs(rho) <= 1.0e-30) return FLURSYS_ERR_BREAKDOWN;
        double beta = (rho / rho_prev) * (alpha / omega);
        if (!std::isfinite(beta)) return FLURSYS_ERR_BREAKDOWN;
        for (int64_t i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        if ((st = spmv(a, p.data(), v.data()))) return st;
        double den = sdot(rh.data(), v.data(), n);
        if (!std::isfinite(den) || std::fabs(den) <= 1.0e-30) return FLURSYS_ERR_BREAKDOWN;
        alpha = rho / den;
        if (!std::isfinite(alpha)) return FLURSYS_ERR_BREAKDOWN;
        for (int64_t i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
        double sn2 = sdot(s.data(), s.data(), n);
        if (!std::isfinite(sn2)) return FLURSYS_ERR_NON_FINITE;
        double sn = std::sqrt(sn2);
        if (sn <= threshold) {
            for (int64_t i = 0; i < n; ++i) x[i] += alpha * p[i];
            fill_report(rep, FLURSYS_LINEAR_CONVERGED, it, initial, sn);
            return FLURSYS_OK;
        }
        if ((st = spmv(a, s.data(), t.data()))) return st;
        double tt = sdot(t.data(), t.data(), n);
        if (!std::isfinite(tt) || std::fabs(tt) <= 1.0e-30) return FLURSYS_ERR_BREAKDOWN;
        omega = sdot(t.data(), s.data(), n) / tt;
        if (!std::isfinite(omega) || std::fabs(omega) <= 1.0e-30) return FLURSYS_ERR_BREAKDOWN;
        for (int64_t i = 0; i < n; ++i) {
            x[i] += alpha * p[i] + omega * s[i];
            r[i] = s[i] - omega * t[i];
        }
        double rn2 = sdot(r.data(), r.data(), n);
        if (!std::isfinite(rn2)) return FLURSYS_ERR_NON_FINITE;
        double rn = std::sqrt(rn2);
        if (rn <= threshold) { fill_report(rep, FLURSYS_LINEAR_CONVERGED, it, initial, rn); return FLURSYS_OK; }
        rho_prev = rho;
    }
    double fin = std::sqrt(sdot(r.data(), r.data(), n));
    fill_report(rep, FLURSYS_LINEAR_MAX_ITERATIONS, o.max_iterations, initial, fin);
    return FLURSYS_OK;
}

// SimulationConfig::validate (incompressible.rs:93-191) without thermal
// checks, and LidDrivenCavity3DConfig::validate (incompressible_3d.rs:50-84).
int32_t validate_config(const FlursysCudaConfig &c, std::string *msg) {
    auto fin_pos = [](double x) { return std::isfinite(x) && x > 0.0; };
    if (c.dimension == 3) {
        // src/project.rs:276-284: the 3D backend runs constant-property flow only
        if (c.physics.energy_model != FLURSYS_ENERGY_OFF || c.physics.buoyancy != FLURSYS_BUOYANCY_OFF) { *msg = "the current 3D backend supports constant-property flow only; thermal and buoyancy models are not available"; return FLURSYS_ERR_UNSUPPORTED; }
        if (c.nx < 4 || c.ny < 4 || c.nz < 4) { *msg = "nx, ny, and nz must all be at least 4"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!(c.case_params.length > 0.0 && c.case_params.height > 0.0 && c.case_params.depth > 0.0)) { *msg = "Domain dimensions must be positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!fin_pos(c.case_params.density)) { *msg = "density must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!fin_pos(c.case_params.reference_velocity)) { *msg = "lid_velocity must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!fin_pos(c.case_params.reynolds)) { *msg = "reynolds must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!fin_pos(c.dt)) { *msg = "dt must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (c.max_steps <= 0 || c.pressure_max_iters <= 0) { *msg = "iteration limits must be positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!fin_pos(c.pressure_tolerance)) { *msg = "pressure_tolerance must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!(std::isfinite(c.pressure_omega) && c.pressure_omega > 0.0 && c.pressure_omega < 2.0)) { *msg = "pressure_omega must lie between 0 and 2"; return FLURSYS_ERR_INVALID_CONFIG; }
        return FLURSYS_OK;
    }
    if (c.dimension != 2) { *msg = "dimension must be 2 or 3"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (c.nx < 4 || c.ny < 4) { *msg = "nx and ny must be at least 4"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (!fin_pos(c.dt)) { *msg = "dt must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (!std::isfinite(c.t_end) || c.t_end < 0.0) { *msg = "t_end must be finite and non-negative"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (c.coupling == FLURSYS_COUPLING_PROJECTION && c.t_end == 0.0) { *msg = "t_end must be positive for projection coupling"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (c.max_steps <= 0) { *msg = "max_steps must be positive"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (c.pressure_max_iters <= 0) { *msg = "pressure_max_iters must be positive"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (!std::isfinite(c.pressure_omega) || c.pressure_omega <= 0.0 || c.pressure_omega >= 2.0) { *msg = "pressure_omega must lie between 0 and 2"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (!std::isfinite(c.velocity_relaxation) || c.velocity_relaxation <= 0.0 || c.velocity_relaxation > 1.0) { *msg = "velocity_relaxation must lie between 0 (exclusive) and 1"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (!std::isfinite(c.pressure_relaxation) || c.pressure_relaxation <= 0.0 || c.pressure_relaxation > 1.0) { *msg = "pressure_relaxation must lie between 0 (exclusive) and 1"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (!fin_pos(c.steady_tolerance)) { *msg = "steady_tolerance must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (!fin_pos(c.case_params.density) || !fin_pos(c.case_params.kinematic_viscosity)) { *msg = "fluid density and kinematic viscosity must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
    if (c.adaptive) {
        if (c.coupling != FLURSYS_COUPLING_PROJECTION) { *msg = "adaptive time stepping requires transient projection coupling"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!fin_pos(c.min_dt)) { *msg = "adaptive min_dt must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!fin_pos(c.max_dt)) { *msg = "adaptive max_dt must be finite and positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (c.min_dt > c.max_dt) { *msg = "adaptive min_dt must not exceed max_dt"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (c.dt < c.min_dt || c.dt > c.max_dt) { *msg = "adaptive initial dt must lie between min_dt and max_dt"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!std::isfinite(c.target_cfl) || c.target_cfl <= 0.0 || c.target_cfl > 1.0) { *msg = "adaptive target_cfl must lie between 0 (exclusive) and 1"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!std::isfinite(c.target_diffusion_number) || c.target_diffusion_number <= 0.0 || c.target_diffusion_number > 0.5) { *msg = "adaptive target_diffusion_number must lie between 0 (exclusive) and 0.5"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!std::isfinite(c.max_growth_factor) || c.max_growth_factor < 1.0) { *msg = "adaptive max_growth_factor must be finite and at least 1"; return FLURSYS_ERR_INVALID_CONFIG; }
    }
    if (!(c.case_params.length > 0.0 && c.case_params.height > 0.0)) { *msg = "Domain dimensions must be positive"; return FLURSYS_ERR_INVALID_CONFIG; }
    // PhysicsSettings::validate (src/physics.rs:79-131) at min_dt when
    // adaptive, else dt (incompressible.rs:180-189)
    const FlursysPhysicsSettings &ph = c.physics;
    const bool thermal = ph.energy_model == FLURSYS_ENERGY_CONSTANT_PROPERTIES;
    if (thermal) {
        if (!std::isfinite(ph.initial_temperature) || !std::isfinite(ph.thermal_diffusivity) || ph.thermal_diffusivity <= 0.0 || !std::isfinite(ph.source_temperature_rate)) { *msg = "thermal initial temperature, diffusivity, and source must be finite; diffusivity must be positive"; return FLURSYS_ERR_INVALID_CONFIG; }
        for (int s = 0; s < 4; ++s)
            if (ph.thermal[s].kind == FLURSYS_THERMAL_FIXED_TEMPERATURE && !std::isfinite(ph.thermal[s].temperature)) { *msg = "fixed thermal boundary temperatures must be finite"; return FLURSYS_ERR_INVALID_CONFIG; }
        const double vdt = c.adaptive ? c.min_dt : c.dt;
        const double dx = c.case_params.length / c.nx, dy = c.case_params.height / c.ny;
        const double fourier = ph.thermal_diffusivity * vdt * (std::pow(1.0 / dx, 2) + std::pow(1.0 / dy, 2));
        if (fourier > 0.5) { *msg = "explicit thermal diffusion is unstable: alpha*dt*(1/dx^2 + 1/dy^2)=" + rust_sci(fourier, 3) + " exceeds 0.5"; return FLURSYS_ERR_INVALID_CONFIG; }
    }
    if (ph.buoyancy == FLURSYS_BUOYANCY_BOUSSINESQ) {
        if (!thermal) { *msg = "Boussinesq buoyancy requires the constant-property energy equation"; return FLURSYS_ERR_INVALID_CONFIG; }
        if (!std::isfinite(ph.reference_temperature) || !std::isfinite(ph.thermal_expansion) || ph.thermal_expansion < 0.0 || !std::isfinite(ph.gravity_x) || !std::isfinite(ph.gravity_y)) { *msg = "Boussinesq reference temperature, expansion coefficient, and gravity must be finite; expansion must be non-negative"; return FLURSYS_ERR_INVALID_CONFIG; }
    }
    return FLURSYS_OK;
}

}  // namespace

// ===========================================================================
// C API
// ===========================================================================
extern "C" {

void orc_set_threads(int32_t threads) { g_threads = threads < 1 ? 1 : threads; }
int32_t orc_get_threads(void) { return g_threads; }

int32_t orc_csr_validate(int64_t nrows, int64_t ncols, int64_t nnz, const int64_t *ro, const int64_t *ci,
                         const double *v, char *msg, size_t msg_size) {
    std::string m;
    int32_t st = validate_csr(nrows, ncols, nnz, ro, ci, v, &m);
    copy_msg(m, msg, msg_size);
    return st;
}

// CsrBuilder::add + finalize (csr.rs:131-192)
int32_t orc_csr_build(int64_t nrows, int64_t ncols, int64_t nentries, const int64_t *rows,
                      const int64_t *cols, const double *vals, int64_t *ro_out, int64_t *ci_out,
                      double *v_out, int64_t *nnz_out) {
    std::vector<std::tuple<int64_t, int64_t, double>> e;
    e.reserve(nentries);
    for (int64_t k = 0; k < nentries; ++k) {
        if (rows[k] < 0 || rows[k] >= nrows || cols[k] < 0 || cols[k] >= ncols) return FLURSYS_ERR_INDEX_OUT_OF_BOUNDS;
        if (!std::isfinite(vals[k])) return FLURSYS_ERR_NON_FINITE;
        e.emplace_back(rows[k], cols[k], vals[k]);
    }
    // The reference sorts by (row, column) with an unstable sort and then sums
    // duplicates in sorted order; duplicates of one (row, column) are summed
    // in insertion order here (stable sort), which equals the reference's sum
    // up to rounding when there are three or more duplicates.
    std::stable_sort(e.begin(), e.end(), [](const auto &a, const auto &b) {
        return std::get<0>(a) != std::get<0>(b) ? std::get<0>(a) < std::get<0>(b) : std::get<1>(a) < std::get<1>(b);
    });
    int64_t nnz = 0;
    size_t k = 0;
    ro_out[0] = 0;
    for (int64_t r = 0; r < nrows; ++r) {
        while (k < e.size() && std::get<0>(e[k]) == r) {
            int64_t col = std::get<1>(e[k]);
            double s = 0.0;
            while (k < e.size() && std::get<0>(e[k]) == r && std::get<1>(e[k]) == col) s += std::get<2>(e[k++]);
            if (!std::isfinite(s)) return FLURSYS_ERR_NON_FINITE;
            if (s != 0.0) { ci_out[nnz] = col; v_out[nnz] = s; ++nnz; }
        }
        ro_out[r + 1] = nnz;
    }
    *nnz_out = nnz;
    return FLURSYS_OK;
}

int32_t orc_csr_spmv(int64_t nrows, int64_t ncols, int64_t nnz, const int64_t *ro, const int64_t *ci,
                     const double *v, const double *input, double *output) {
    std::string m;
    int32_t st = validate_csr(nrows, ncols, nnz, ro, ci, v, &m);
    if (st) return st;
    Csr a{nrows, ncols, ro, ci, v};
    return spmv(a, input, output);
}

int32_t orc_jacobi_inverse_diagonal(int64_t n, int64_t nnz, const int64_t *ro, const int64_t *ci,
                                    const double *v, double *inv_out, int64_t *bad_row) {
    (void)nnz;
    Csr a{n, n, ro, ci, v};
    std::vector<double> inv;
    int64_t bad = -1;
    int32_t st = jacobi(a, inv, &bad);
    if (bad_row) *bad_row = bad;
    if (st) return st;
    std::memcpy(inv_out, inv.data(), n * sizeof(double));
    return FLURSYS_OK;
}

int32_t orc_csr_solve(int32_t method, int64_t n, int64_t nnz, const int64_t *ro, const int64_t *ci,
                      const double *v, const double *rhs, double *x, const FlursysLinearSolverOptions *o,
                      FlursysLinearSolveReport *rep) {
    std::string m;
    int32_t st = validate_csr(n, n, nnz, ro, ci, v, &m);
    if (st) return st;
    Csr a{n, n, ro, ci, v};
    FlursysLinearSolverOptions opt = o ? *o : FlursysLinearSolverOptions{1e-10, 1e-8, 1000};
    if (method == 2) return solve_bicgstab(a, rhs, x, opt, rep);
    if (method == 1) {
        std::vector<double> inv;
        int64_t bad = -1;
        if ((st = jacobi(a, inv, &bad))) return st;
        return solve_cg(a, rhs, x, opt, &inv, rep);
    }
    return solve_cg(a, rhs, x, opt, nullptr, rep);
}

void orc_momentum_stability_numbers(double dt, double nu, double dx, double dy, double mu, double mv,
                                    double *cfl, double *dnu) {
    *cfl = dt * (mu / dx + mv / dy);
    *dnu = nu * dt * (1.0 / (dx * dx) + 1.0 / (dy * dy));
}

int32_t orc_adaptive_time_step(double current_dt, double mu, double mv, double dx, double dy, double nu,
                               double thermal, double min_dt, double max_dt, double target_cfl,
                               double target_diff, double growth, double *dt_out, char *msg, size_t msg_size) {
    std::string e;
    int32_t st = adaptive_dt(current_dt, mu, mv, dx, dy, nu, thermal, min_dt, max_dt, target_cfl, target_diff,
                             growth, dt_out, &e);
    copy_msg(e, msg, msg_size);
    return st;
}

// Defaults: LidDrivenCavity3DConfig::default() (incompressible_3d.rs:27-47)
// and the CLI cavity defaults (src/bin/flursys.rs:102-123,236-300).
int32_t orc_default_config(int32_t dimension, FlursysCudaConfig *c) {
    if (!c) return FLURSYS_ERR_INVALID_ARGUMENT;
    std::memset(c, 0, sizeof *c);
    c->abi_version = FLURSYS_CUDA_ABI_VERSION;
    c->dimension = dimension == 3 ? 3 : 2;
    c->case_params.kind = FLURSYS_CASE_CAVITY;
    c->case_params.length = 1.0;
    c->case_params.height = 1.0;
    c->case_params.depth = 1.0;
    c->case_params.density = 1.0;
    c->case_params.reference_velocity = 1.0;
    c->case_params.reynolds = 100.0;
    c->case_params.kinematic_viscosity = 0.01;
    c->min_dt = 1.0e-6;
    c->max_dt = 1.0e-2;
    c->target_cfl = 0.5;
    c->target_diffusion_number = 0.25;
    c->max_growth_factor = 1.1;
    c->pressure_solver = FLURSYS_PRESSURE_PCG;
    c->pressure_atol = 0.0;
    c->pressure_rtol = 1.0e-8;
    c->precision = FLURSYS_PRECISION_F64;
    c->residual_replacement_every = 50;
    // ThermalSettings::default (src/physics.rs:43-56); buoyancy off
    c->physics.initial_temperature = 293.15;
    c->physics.thermal_diffusivity = 2.2e-5;
    if (c->dimension == 3) {
        c->nx = c->ny = c->nz = 32;
        c->dt = 5.0e-4;
        c->max_steps = 10000;
        c->pressure_max_iters = 2000;
        c->pressure_tolerance = 1.0e-6;
        c->pressure_omega = 1.7;
        c->pressure_solver = FLURSYS_PRESSURE_SOR;
        c->stop_rule = FLURSYS_STOP_REFERENCE_RESIDUAL;
        c->convection = FLURSYS_CONVECTION_CENTRAL;
        c->t_end = 1e300;
    } else {
        c->nx = c->ny = 64;
        c->nz = 1;
        c->dt = 0.001;
        c->t_end = 100.0;
        c->max_steps = 100000;
        c->convection = FLURSYS_CONVECTION_UPWIND;
        c->coupling = FLURSYS_COUPLING_PROJECTION;
        c->stop_rule = FLURSYS_STOP_ABS_INF;
        c->pressure_max_iters = 1200;
        c->pressure_tolerance = 1.0e-5;
        c->pressure_omega = 1.7;
        c->velocity_relaxation = 0.7;
        c->pressure_relaxation = 0.3;
        c->steady_tolerance = 1.0e-7;
        c->minimum_steps = 2000;
    }
    return FLURSYS_OK;
}

int32_t orc_create(const FlursysCudaConfig *cfg, OracleSolver **out, char *msg, size_t msg_size) {
    if (!cfg || !out) return FLURSYS_ERR_INVALID_ARGUMENT;
    std::string m;
    int32_t st = validate_config(*cfg, &m);
    if (st) {
        copy_msg(m, msg, msg_size);
        return st;
    }
    if (cfg->dimension == 3) *out = new Solver3D(*cfg);
    else *out = new Solver2D(*cfg);
    return FLURSYS_OK;
}

int32_t orc_step(OracleSolver *s, int64_t nsteps, FlursysStepReport *rep) {
    if (!s) return FLURSYS_ERR_INVALID_ARGUMENT;
    for (int64_t n = 0; n < nsteps; ++n) {
        int32_t st = s->advance(rep);
        if (st) return st;
        if (rep && s->cfg.dimension == 2 && (rep->converged || rep->reached_end_time)) break;
    }
    return FLURSYS_OK;
}

size_t orc_field_size(const OracleSolver *s, int32_t id) {
    auto *f = const_cast<OracleSolver *>(s)->field(id);
    return f ? f->size() : 0;
}
int32_t orc_get_field(const OracleSolver *s, int32_t id, double *out, size_t n) {
    auto *f = const_cast<OracleSolver *>(s)->field(id);
    if (!f) return FLURSYS_ERR_INVALID_ARGUMENT;
    if (f->size() != n) return FLURSYS_ERR_DIMENSION_MISMATCH;
    std::memcpy(out, f->data(), n * sizeof(double));
    return FLURSYS_OK;
}
int32_t orc_set_field(OracleSolver *s, int32_t id, const double *in, size_t n) {
    auto *f = s->field(id);
    if (!f) return FLURSYS_ERR_INVALID_ARGUMENT;
    if (f->size() != n) return FLURSYS_ERR_DIMENSION_MISMATCH;
    std::memcpy(f->data(), in, n * sizeof(double));
    return FLURSYS_OK;
}
int32_t orc_last_error(const OracleSolver *s, char *buf, size_t size) {
    copy_msg(s ? s->err : std::string(), buf, size);
    return FLURSYS_OK;
}
void orc_destroy(OracleSolver *s) { delete s; }

int32_t orc_phase_predict(OracleSolver *s, double dt) { return s->predict(dt); }
int32_t orc_phase_rhs(OracleSolver *s, double dt) { return s->rhs_phase(dt); }
int32_t orc_phase_pressure(OracleSolver *s, double *res, int64_t *its) { return s->pressure(res, its); }
int32_t orc_phase_correct(OracleSolver *s, double dt) { return s->correct(dt); }
double orc_max_divergence(const OracleSolver *s) { return s->max_divergence(); }
double orc_pressure_residual(const OracleSolver *s) { return s->pressure_residual(); }
double orc_max_speed(const OracleSolver *s) { return s->max_speed(); }

int32_t orc_stencil_pcg(int64_t nx, int64_t ny, int64_t nz, double dx, double dy, double dz,
                        const double *rhs, double *x_inout, const FlursysLinearSolverOptions *o,
                        FlursysLinearSolveReport *rep) {
    if (nx < 1 || ny < 1 || nz < 1 || !rhs || !x_inout || !o) return FLURSYS_ERR_INVALID_ARGUMENT;
    const int64_t n = nx * ny * nz;
    std::vector<double> b(n), x(x_inout, x_inout + n);
    for (int64_t k = 0; k < n; ++k) b[k] = -rhs[k];
    StopRule stop;
    stop.rule = FLURSYS_STOP_REL_L2;
    stop.atol = o->absolute_tolerance;
    stop.rtol = o->relative_tolerance;
    PcgResult r;
    if (nz == 1) {
        Neumann2DOperator op(nx, ny, dx, dy);
        r = pcg_core(op, b, x, stop, o->max_iterations);
    } else {
        Pinned3DOperator op(nx, ny, nz, dx, dy, dz);
        b[0] = 0.0;
        x[0] = 0.0;
        r = pcg_core(op, b, x, stop, o->max_iterations);
    }
    if (r.status) return r.status;
    std::memcpy(x_inout, x.data(), n * sizeof(double));
    fill_report(rep, r.linear_status, r.iterations, r.initial, r.residual);
    return FLURSYS_OK;
}

}  // extern "C"

// ===========================================================================
// Steady collocated SIMPLE (src/simple.rs, src/momentum.rs, src/numerics.rs,
// src/unstructured_incompressible.rs) on a general face-based mesh, here
// built for the uniform quad channel. FP64, serial, reference loop order.
// ===========================================================================
namespace {

struct V3 {
    double x = 0.0, y = 0.0, z = 0.0;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

enum Patch : int { kInternal = -1, kInlet = 0, kOutlet = 1, kBottom = 2, kTop = 3 };

// UnstructuredMesh (src/mesh.rs:201-230) for a 2D quad grid with unit depth:
// face area vector = edge rotated outward from the owner, |S| = edge length,
// cell volume = cell area (mesh.rs:563-616).
struct FvMesh {
    int64_t nx = 0, ny = 0;
    std::vector<V3> cc;               // cell centres
    std::vector<double> vol;
    std::vector<int64_t> owner, neigh;  // neigh -1 on boundary faces
    std::vector<V3> area, fc;
    std::vector<int> patch;
    std::vector<std::vector<int64_t>> cell_faces;
    int64_t ncells() const { return (int64_t)cc.size(); }
    int64_t nfaces() const { return (int64_t)owner.size(); }
};

FvMesh channel_mesh(int64_t nx, int64_t ny, double L, double H) {
    FvMesh m;
    m.nx = nx;
    m.ny = ny;
    const double dx = L / nx, dy = H / ny;
    m.cc.resize(nx * ny);
    m.vol.assign(nx * ny, dx * dy);
    m.cell_faces.resize(nx * ny);
    for (int64_t j = 0; j < ny; ++j)
        for (int64_t i = 0; i < nx; ++i) m.cc[i + nx * j] = {(i + 0.5) * dx, (j + 0.5) * dy, 0.0};
    auto add = [&](int64_t o, int64_t n, V3 s, V3 c, int p) {
        m.owner.push_back(o);
        m.neigh.push_back(n);
        m.area.push_back(s);
        m.fc.push_back(c);
        m.patch.push_back(p);
        const int64_t f = m.nfaces() - 1;
        m.cell_faces[o].push_back(f);
        if (n >= 0) m.cell_faces[n].push_back(f);
    };
    for (int64_t j = 0; j < ny; ++j)
        for (int64_t i = 0; i + 1 < nx; ++i)
            add(i + nx * j, i + 1 + nx * j, {dy, 0, 0}, {(i + 1) * dx, (j + 0.5) * dy, 0}, kInternal);
    for (int64_t j = 0; j + 1 < ny; ++j)
        for (int64_t i = 0; i < nx; ++i)
            add(i + nx * j, i + nx * (j + 1), {0, dx, 0}, {(i + 0.5) * dx, (j + 1) * dy, 0}, kInternal);
    for (int64_t j = 0; j < ny; ++j) add(nx * j, -1, {-dy, 0, 0}, {0.0, (j + 0.5) * dy, 0}, kInlet);
    for (int64_t j = 0; j < ny; ++j) add(nx - 1 + nx * j, -1, {dy, 0, 0}, {L, (j + 0.5) * dy, 0}, kOutlet);
    for (int64_t i = 0; i < nx; ++i) add(i, -1, {0, -dx, 0}, {(i + 0.5) * dx, 0.0, 0}, kBottom);
    for (int64_t i = 0; i < nx; ++i) add(i + nx * (ny - 1), -1, {0, dx, 0}, {(i + 0.5) * dx, H, 0}, kTop);
    return m;
}

// ScalarBoundaryCondition per face (numerics.rs): fixed value or zero gradient.
struct ScalarBc {
    std::vector<int> fixed;  // 1 FixedValue, 0 ZeroGradient (boundary faces)
    std::vector<double> value;
};

// weight (numerics.rs:294-303)
double iweight(const FvMesh &m, int64_t f) {
    const V3 d = m.cc[m.neigh[f]] - m.cc[m.owner[f]];
    return dot(m.fc[f] - m.cc[m.owner[f]], d) / dot(d, d);
}

// LeastSquaresGradientStencil::new (numerics.rs:106-200), 2D.
struct LsEq {
    V3 coef;
    int64_t nb;   // neighbour cell, or -1 for a fixed boundary value
    double value;
};
struct LsStencil {
    std::vector<std::vector<LsEq>> eqs;
    std::vector<std::array<double, 9>> inv;
};

int32_t ls_stencil(const FvMesh &m, const ScalarBc &bc, LsStencil *out) {
    out->eqs.assign(m.ncells(), {});
    out->inv.assign(m.ncells(), {});
    for (int64_t c = 0; c < m.ncells(); ++c) {
        double nm[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int64_t f : m.cell_faces[c]) {
            V3 off;
            LsEq e{};
            if (m.neigh[f] >= 0) {
                const int64_t nb = m.owner[f] == c ? m.neigh[f] : m.owner[f];
                off = m.cc[nb] - m.cc[c];
                e.nb = nb;
            } else {
                if (!bc.fixed[f]) continue;  // zero gradient: no equation in 2D
                off = m.fc[f] - m.cc[c];
                e.nb = -1;
                e.value = bc.value[f];
            }
            const double w = 1.0 / dot(off, off);
            const V3 rc = off * w;
            nm[0] += rc.x * off.x; nm[1] += rc.x * off.y; nm[2] += rc.x * off.z;
            nm[3] += rc.y * off.x; nm[4] += rc.y * off.y; nm[5] += rc.y * off.z;
            nm[6] += rc.z * off.x; nm[7] += rc.z * off.y; nm[8] += rc.z * off.z;
            e.coef = rc;
            out->eqs[c].push_back(e);
        }
        // inverse_normal_matrix, TwoD (numerics.rs:236-254)
        const double det = nm[0] * nm[4] - nm[1] * nm[3];
        const double scale = std::max(std::max(std::fabs(nm[0]), std::fabs(nm[4])), 1.0);
        if (std::fabs(det) <= 2.220446049250313e-16 * scale * scale) return FLURSYS_ERR_BREAKDOWN;
        out->inv[c] = {nm[4] / det, -nm[1] / det, 0.0, -nm[3] / det, nm[0] / det, 0.0, 0.0, 0.0, 0.0};
    }
    return FLURSYS_OK;
}

// least_squares_gradient_into (numerics.rs:650-682)
std::vector<V3> ls_gradient(const LsStencil &s, const std::vector<double> &v) {
    std::vector<V3> g(v.size());
    for (size_t c = 0; c < v.size(); ++c) {
        V3 r;
        for (const LsEq &e : s.eqs[c]) {
            const double adj = e.nb >= 0 ? v[e.nb] : e.value;
            r = r + e.coef * (adj - v[c]);
        }
        const auto &I = s.inv[c];
        g[c] = {I[0] * r.x + I[1] * r.y + I[2] * r.z, I[3] * r.x + I[4] * r.y + I[5] * r.z,
                I[6] * r.x + I[7] * r.y + I[8] * r.z};
    }
    return g;
}

// CsrBuilder::add + finalize (csr.rs:131-192) into owned arrays.
struct OwnedCsr {
    int64_t n = 0;
    std::vector<int64_t> ro, ci;
    std::vector<double> v;
    Csr view() const { return Csr{n, n, ro.data(), ci.data(), v.data()}; }
    double diag(int64_t r) const {
        for (int64_t e = ro[r]; e < ro[r + 1]; ++e)
            if (ci[e] == r) return v[e];
        return 0.0;
    }
};

int32_t build_csr(int64_t n, const std::vector<std::tuple<int64_t, int64_t, double>> &entries, OwnedCsr *out) {
    std::vector<int64_t> rows(entries.size()), cols(entries.size());
    std::vector<double> vals(entries.size());
    for (size_t k = 0; k < entries.size(); ++k) {
        rows[k] = std::get<0>(entries[k]);
        cols[k] = std::get<1>(entries[k]);
        vals[k] = std::get<2>(entries[k]);
    }
    out->n = n;
    out->ro.assign(n + 1, 0);
    out->ci.assign(entries.size(), 0);
    out->v.assign(entries.size(), 0.0);
    int64_t nnz = 0;
    int32_t st = orc_csr_build(n, n, (int64_t)entries.size(), rows.data(), cols.data(), vals.data(), out->ro.data(),
                               out->ci.data(), out->v.data(), &nnz);
    out->ci.resize(nnz);
    out->v.resize(nnz);
    return st;
}

// assemble_momentum_component (momentum.rs:180-341): upwind convection,
// two-point diffusion, explicit source, equation under-relaxation.
int32_t assemble_momentum(const FvMesh &m, double nu, const ScalarBc &bc, const std::vector<double> &flux,
                          const std::vector<double> &source, const std::vector<double> &current, double alpha,
                          OwnedCsr *A, std::vector<double> *rhs_out) {
    const int64_t n = m.ncells();
    std::vector<std::tuple<int64_t, int64_t, double>> e;
    e.reserve(m.nfaces() * 4 + n);
    std::vector<double> rhs(n, 0.0);
    for (int64_t c = 0; c < n; ++c) rhs[c] += source[c] * m.vol[c];
    for (int64_t f = 0; f < m.nfaces(); ++f) {
        const double phi = flux[f];
        const int64_t o = m.owner[f];
        if (m.neigh[f] >= 0) {
            const int64_t nb = m.neigh[f];
            const V3 d = m.cc[nb] - m.cc[o];
            const double D = nu * dot(m.area[f], d) / dot(d, d);
            e.emplace_back(o, o, D + std::max(phi, 0.0));
            e.emplace_back(o, nb, -D + std::min(phi, 0.0));
            e.emplace_back(nb, o, -D - std::max(phi, 0.0));
            e.emplace_back(nb, nb, D - std::min(phi, 0.0));
        } else {
            const V3 d = m.fc[f] - m.cc[o];
            const double D = nu * dot(m.area[f], d) / dot(d, d);
            if (bc.fixed[f]) {
                const double val = bc.value[f];
                e.emplace_back(o, o, D + std::max(phi, 0.0));
                rhs[o] += D * val - std::min(phi, 0.0) * val;
            } else {
                if (phi < 0.0) return FLURSYS_ERR_INVALID_CONFIG;  // BackflowOnZeroGradient
                e.emplace_back(o, o, phi);
            }
        }
    }
    OwnedCsr un;
    int32_t st = build_csr(n, e, &un);
    if (st) return st;
    if (alpha == 1.0) {
        *A = std::move(un);
        *rhs_out = std::move(rhs);
        return FLURSYS_OK;
    }
    std::vector<std::tuple<int64_t, int64_t, double>> r;
    r.reserve(un.v.size());
    for (int64_t row = 0; row < n; ++row) {
        const double dg = un.diag(row);
        for (int64_t k = un.ro[row]; k < un.ro[row + 1]; ++k) {
            double v = un.v[k];
            if (un.ci[k] == row) v /= alpha;
            r.emplace_back(row, un.ci[k], v);
        }
        rhs[row] += (1.0 - alpha) / alpha * dg * current[row];
    }
    st = build_csr(n, r, A);
    *rhs_out = std::move(rhs);
    return st;
}

struct SimpleOut {
    std::vector<double> u, v, p, flux, history;
    FlursysSimpleReport rep{};
};

// pressure_face_coefficients[_with_boundary] (simple.rs:342-410): rAU
// interpolated to internal faces times (S.d)/(d.d); fixed correction faces
// (pcbc != null) take rAU_P (S.d)/(d.d) with d from the owner to the face.
int32_t pressure_face_coefficients(const FvMesh &m, const std::vector<double> &rau, const ScalarBc *pcbc,
                                   std::vector<double> *coef) {
    coef->assign(m.nfaces(), 0.0);
    for (int64_t f = 0; f < m.nfaces(); ++f) {
        const int64_t o = m.owner[f];
        double c;
        if (m.neigh[f] >= 0) {
            const int64_t nb = m.neigh[f];
            const V3 d = m.cc[nb] - m.cc[o];
            const double d2 = dot(d, d);
            if (!std::isfinite(d2) || d2 <= 2.220446049250313e-16) return FLURSYS_ERR_INVALID_CONFIG;
            const double l = iweight(m, f);
            c = (rau[o] * (1.0 - l) + rau[nb] * l) * dot(m.area[f], d) / d2;
        } else if (pcbc && pcbc->fixed[f]) {
            const V3 d = m.fc[f] - m.cc[o];
            const double d2 = dot(d, d);
            if (!std::isfinite(d2) || d2 <= 2.220446049250313e-16) return FLURSYS_ERR_INVALID_CONFIG;
            c = rau[o] * dot(m.area[f], d) / d2;
        } else {
            continue;
        }
        if (!std::isfinite(c) || c <= 0.0) return FLURSYS_ERR_INVALID_CONFIG;  // InvalidPressureFaceCoefficient
        (*coef)[f] = c;
    }
    return FLURSYS_OK;
}

// correct_face_flux[_with_boundary] (simple.rs:412-496):
// Phi = Phi* - d_f (p'_N - p'_P) on internal faces and, with pcbc, on fixed
// correction faces with p'_b in place of p'_N.
int32_t correct_face_flux(const FvMesh &m, const std::vector<double> &pf, const std::vector<double> &coef,
                          const std::vector<double> &pc, const ScalarBc *pcbc, std::vector<double> *out) {
    *out = pf;
    for (int64_t f = 0; f < m.nfaces(); ++f) {
        double other;
        if (m.neigh[f] >= 0) other = pc[m.neigh[f]];
        else if (pcbc && pcbc->fixed[f]) other = pcbc->value[f];
        else continue;
        const double c = coef[f];
        if (!std::isfinite(c) || c <= 0.0) return FLURSYS_ERR_INVALID_CONFIG;
        (*out)[f] -= c * (other - pc[m.owner[f]]);
        if (!std::isfinite((*out)[f])) return FLURSYS_ERR_INVALID_CONFIG;
    }
    return FLURSYS_OK;
}

// assemble_pressure_correction (simple.rs:518-581, reference cell: its row
// and column are eliminated, rhs 0, diagonal 1) or, with pcbc,
// assemble_pressure_correction_with_boundary (:583-643).
int32_t assemble_pressure_correction(const FvMesh &m, const std::vector<double> &pf, const std::vector<double> &coef,
                                     const ScalarBc *pcbc, int64_t reference_cell, OwnedCsr *P,
                                     std::vector<double> *rhs_out) {
    const int64_t n = m.ncells();
    std::vector<double> rhs(n, 0.0);
    std::vector<std::tuple<int64_t, int64_t, double>> pe;
    pe.reserve(m.nfaces() * 4 + 1);
    bool anchored = false;
    if (!pcbc && (reference_cell < 0 || reference_cell >= n)) return FLURSYS_ERR_INVALID_CONFIG;
    for (int64_t f = 0; f < m.nfaces(); ++f) {
        const double flux = pf[f];
        if (!std::isfinite(flux)) return FLURSYS_ERR_INVALID_CONFIG;
        const int64_t o = m.owner[f];
        rhs[o] -= flux;
        if (m.neigh[f] >= 0) {
            const int64_t nb = m.neigh[f];
            rhs[nb] += flux;
            const double c = coef[f];
            if (!std::isfinite(c) || c <= 0.0) return FLURSYS_ERR_INVALID_CONFIG;
            pe.emplace_back(o, o, c);
            pe.emplace_back(o, nb, -c);
            pe.emplace_back(nb, o, -c);
            pe.emplace_back(nb, nb, c);
        } else if (pcbc && pcbc->fixed[f]) {
            const double c = coef[f], val = pcbc->value[f];
            if (!std::isfinite(c) || c <= 0.0 || !std::isfinite(val)) return FLURSYS_ERR_INVALID_CONFIG;
            pe.emplace_back(o, o, c);
            rhs[o] += c * val;
            anchored = true;
        }
    }
    if (pcbc) {
        if (!anchored) return FLURSYS_ERR_INVALID_CONFIG;  // InvalidPressureReference
    } else {
        std::vector<std::tuple<int64_t, int64_t, double>> kept;
        kept.reserve(pe.size() + 1);
        for (const auto &t : pe)
            if (std::get<0>(t) != reference_cell && std::get<1>(t) != reference_cell) kept.push_back(t);
        rhs[reference_cell] = 0.0;
        kept.emplace_back(reference_cell, reference_cell, 1.0);
        pe.swap(kept);
    }
    int32_t st = build_csr(n, pe, P);
    *rhs_out = std::move(rhs);
    return st;
}

// continuity_rms (simple.rs:706-718): RMS of the integrated cell imbalance.
double continuity_rms(const FvMesh &m, const std::vector<double> &flux) {
    std::vector<double> div(m.ncells(), 0.0);
    for (int64_t f = 0; f < m.nfaces(); ++f) {
        div[m.owner[f]] += flux[f];
        if (m.neigh[f] >= 0) div[m.neigh[f]] -= flux[f];
    }
    double s = 0.0;
    for (double d : div) s += d * d;
    return std::sqrt(s / double(m.ncells()));
}

// correct_cell_velocity_from_gradient (simple.rs:673-704): U = U* - rAU grad p'.
int32_t correct_cell_velocity(const std::vector<V3> &pred, const std::vector<double> &rau,
                              const std::vector<V3> &grad, std::vector<V3> *out) {
    out->resize(pred.size());
    for (size_t c = 0; c < pred.size(); ++c) {
        if (!std::isfinite(rau[c]) || rau[c] <= 0.0) return FLURSYS_ERR_INVALID_CONFIG;  // InvalidMomentumDiagonal
        const V3 v = pred[c] - grad[c] * rau[c];
        if (!(std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z))) return FLURSYS_ERR_INVALID_CONFIG;
        (*out)[c] = v;
    }
    return FLURSYS_OK;
}

// initial_face_flux (simple.rs:724-755): internal faces from the
// geometrically interpolated cell velocity, boundary faces from wall_flux.
std::vector<double> initial_face_flux(const FvMesh &m, const std::vector<V3> &U, const std::vector<double> &wall) {
    std::vector<double> flux = wall;
    for (int64_t f = 0; f < m.nfaces(); ++f)
        if (m.neigh[f] >= 0) {
            const double l = iweight(m, f);
            flux[f] = dot(U[m.owner[f]] * (1.0 - l) + U[m.neigh[f]] * l, m.area[f]);
        }
    return flux;
}

// Steady SIMPLE on a face-based mesh: boundary conditions per face for the
// velocity components and the pressure (the least-squares stencil), and an
// optional pressure-correction boundary (fixed faces anchor the system,
// otherwise `reference_cell` does).
struct SimpleSetup {
    ScalarBc vel[3], pbc;
    const ScalarBc *pcbc = nullptr;
    int64_t reference_cell = 0;
    double nu = 0.0, velocity_relaxation = 0.7, pressure_relaxation = 0.3;
    int64_t max_outer = 1;
    double continuity_tolerance = 0.0;
    FlursysLinearSolverOptions momentum_solver{}, pressure_solver{};
};

// solve_simple (simple.rs:148-314). U, p, flux carry the initial state in
// and the result out; `out` receives the history and the report.
int32_t simple_solve(const FvMesh &m, const SimpleSetup &su, std::vector<V3> &U3, std::vector<double> &p,
                     std::vector<double> &flux, SimpleOut *out) {
    const int64_t n = m.ncells(), nf = m.nfaces();
    if (su.max_outer < 1) return FLURSYS_ERR_INVALID_CONFIG;
    if (!(std::isfinite(su.pressure_relaxation) && su.pressure_relaxation > 0.0 && su.pressure_relaxation <= 1.0))
        return FLURSYS_ERR_INVALID_CONFIG;
    if (!(std::isfinite(su.continuity_tolerance) && su.continuity_tolerance >= 0.0)) return FLURSYS_ERR_INVALID_CONFIG;
    LsStencil stencil;
    int32_t st = ls_stencil(m, su.pbc, &stencil);
    if (st) return st;
    out->history.assign(1, continuity_rms(m, flux));
    FlursysSimpleReport &rep = out->rep;
    rep = FlursysSimpleReport{};
    rep.initial_continuity_rms = out->history[0];
    rep.final_continuity_rms = out->history[0];
    for (int64_t it = 1; it <= su.max_outer; ++it) {
        // pressure_gradient_source with unit density
        const std::vector<V3> gp = ls_gradient(stencil, p);
        OwnedCsr A[3];
        std::vector<double> b[3];
        for (int k = 0; k < 3; ++k) {
            std::vector<double> src(n), cur(n);
            for (int64_t c = 0; c < n; ++c) {
                src[c] = -(k == 0 ? gp[c].x : k == 1 ? gp[c].y : gp[c].z);
                cur[c] = k == 0 ? U3[c].x : k == 1 ? U3[c].y : U3[c].z;
            }
            st = assemble_momentum(m, su.nu, su.vel[k], flux, src, cur, su.velocity_relaxation, &A[k], &b[k]);
            if (st) return st;
        }
        // solve_momentum_velocity: BiCGSTAB per component from the current velocity
        std::vector<double> comp[3];
        for (int k = 0; k < 3; ++k) {
            comp[k].resize(n);
            for (int64_t c = 0; c < n; ++c) comp[k][c] = k == 0 ? U3[c].x : k == 1 ? U3[c].y : U3[c].z;
            st = solve_bicgstab(A[k].view(), b[k].data(), comp[k].data(), su.momentum_solver, &rep.momentum[k]);
            if (st) return st;
            if (rep.momentum[k].status != FLURSYS_LINEAR_CONVERGED) return FLURSYS_ERR_BREAKDOWN;
        }
        std::vector<V3> pred(n);
        for (int64_t c = 0; c < n; ++c) pred[c] = {comp[0][c], comp[1][c], comp[2][c]};
        // momentum_inverse_diagonal of the x system (simple.rs:319-332)
        std::vector<double> rau(n);
        for (int64_t c = 0; c < n; ++c) {
            const double d = A[0].diag(c);
            if (!(std::isfinite(d) && d > 0.0)) return FLURSYS_ERR_INVALID_CONFIG;
            rau[c] = 1.0 / d;
        }
        // rhie_chow_predicted_flux (simple.rs:757-805), then the prescribed
        // normal flux of fixed correction faces from the owner's predictor
        std::vector<double> coef_int;
        st = pressure_face_coefficients(m, rau, nullptr, &coef_int);
        if (st) return st;
        std::vector<double> pf = flux;
        for (int64_t f = 0; f < nf; ++f) {
            const int64_t o = m.owner[f];
            if (m.neigh[f] >= 0) {
                const int64_t nb = m.neigh[f];
                const double l = iweight(m, f);
                const V3 fu = pred[o] * (1.0 - l) + pred[nb] * l;
                const V3 fr = gp[o] * rau[o] * (1.0 - l) + gp[nb] * rau[nb] * l;
                pf[f] = dot(fu, m.area[f]) + dot(fr, m.area[f]) - coef_int[f] * (p[nb] - p[o]);
                if (!std::isfinite(pf[f])) return FLURSYS_ERR_INVALID_CONFIG;
            } else if (su.pcbc && su.pcbc->fixed[f]) {
                pf[f] = dot(pred[o], m.area[f]);
            }
        }
        std::vector<double> coef;
        if (su.pcbc) {
            st = pressure_face_coefficients(m, rau, su.pcbc, &coef);
            if (st) return st;
        } else {
            coef = coef_int;
        }
        OwnedCsr P;
        std::vector<double> prhs;
        if ((st = assemble_pressure_correction(m, pf, coef, su.pcbc, su.reference_cell, &P, &prhs))) return st;
        // solve_pressure_correction (simple.rs:648-668): Jacobi-PCG from zero
        std::vector<double> pc(n, 0.0), inv;
        int64_t bad = -1;
        if ((st = jacobi(P.view(), inv, &bad))) return st;
        st = solve_cg(P.view(), prhs.data(), pc.data(), su.pressure_solver, &inv, &rep.pressure);
        if (st) return st;
        if (rep.pressure.status != FLURSYS_LINEAR_CONVERGED) return FLURSYS_ERR_BREAKDOWN;
        for (int64_t c = 0; c < n; ++c) p[c] += su.pressure_relaxation * pc[c];
        const std::vector<V3> gpc = ls_gradient(stencil, pc);
        if ((st = correct_cell_velocity(pred, rau, gpc, &U3))) return st;
        if ((st = correct_face_flux(m, pf, coef, pc, su.pcbc, &flux))) return st;
        const double cont = continuity_rms(m, flux);
        out->history.push_back(cont);
        rep.outer_iterations = it;
        rep.final_continuity_rms = cont;
        if (cont <= su.continuity_tolerance) {
            rep.converged = 1;
            break;
        }
    }
    return FLURSYS_OK;
}

// solve_incompressible for the channel case (unstructured_incompressible.rs:
// 106-212, 368-482): parabolic velocity inlet, fixed-pressure outlet, no-slip
// walls, zero initial state.
int32_t simple_channel(const FlursysSimpleConfig &cfg, SimpleOut *out) {
    const int64_t nx = cfg.nx, ny = cfg.ny;
    if (nx < 2 || ny < 2) return FLURSYS_ERR_INVALID_CONFIG;
    if (cfg.max_outer_iterations < 1) return FLURSYS_ERR_INVALID_CONFIG;
    if (!(cfg.pressure_relaxation > 0.0 && cfg.pressure_relaxation <= 1.0)) return FLURSYS_ERR_INVALID_CONFIG;
    if (!(cfg.velocity_relaxation > 0.0 && cfg.velocity_relaxation <= 1.0)) return FLURSYS_ERR_INVALID_CONFIG;
    const FvMesh m = channel_mesh(nx, ny, cfg.length, cfg.height);
    const int64_t n = m.ncells(), nf = m.nfaces();
    const double H = cfg.height, U = cfg.inlet_peak_velocity;
    SimpleSetup su;
    ScalarBc pcbc;
    for (ScalarBc *b : {&su.vel[0], &su.vel[1], &su.vel[2], &su.pbc, &pcbc}) {
        b->fixed.assign(nf, 0);
        b->value.assign(nf, 0.0);
    }
    std::vector<double> bflux(nf, 0.0);
    for (int64_t f = 0; f < nf; ++f) {
        if (m.patch[f] == kInternal) continue;
        if (m.patch[f] == kOutlet) {
            su.pbc.fixed[f] = 1;
            su.pbc.value[f] = cfg.outlet_pressure;
            pcbc.fixed[f] = 1;
            pcbc.value[f] = 0.0;
            continue;  // velocity zero gradient, no prescribed flux
        }
        V3 u{};
        if (m.patch[f] == kInlet) {
            const double y = m.fc[f].y;
            u.x = U * 4.0 * y * (H - y) / (H * H);
        }
        su.vel[0].fixed[f] = su.vel[1].fixed[f] = su.vel[2].fixed[f] = 1;
        su.vel[0].value[f] = u.x;
        su.vel[1].value[f] = u.y;
        su.vel[2].value[f] = u.z;
        bflux[f] = dot(u, m.area[f]);
    }
    su.pcbc = &pcbc;
    su.nu = cfg.kinematic_viscosity;
    su.velocity_relaxation = cfg.velocity_relaxation;
    su.pressure_relaxation = cfg.pressure_relaxation;
    su.max_outer = cfg.max_outer_iterations;
    su.continuity_tolerance = cfg.continuity_tolerance;
    su.momentum_solver = cfg.momentum_solver;
    su.pressure_solver = cfg.pressure_solver;
    std::vector<V3> U3(n);  // zero initial velocity
    std::vector<double> p(n, 0.0);
    std::vector<double> flux = initial_face_flux(m, U3, bflux);
    int32_t st = simple_solve(m, su, U3, p, flux, out);
    if (st) return st;
    FlursysSimpleReport &rep = out->rep;
    // backflow at the pressure outlet (unstructured_incompressible.rs:430-449)
    for (int64_t f = 0; f < nf; ++f)
        if (m.patch[f] == kOutlet && flux[f] < 0.0) return FLURSYS_ERR_INVALID_CONFIG;
    for (int64_t f = 0; f < nf; ++f) {
        if (m.neigh[f] >= 0) continue;
        if (flux[f] < 0.0) rep.total_inflow += flux[f];
        else rep.total_outflow += flux[f];
    }
    // outputs: cell fields and +x / +y face fluxes
    out->u.resize(n);
    out->v.resize(n);
    out->p = p;
    for (int64_t c = 0; c < n; ++c) {
        out->u[c] = U3[c].x;
        out->v[c] = U3[c].y;
    }
    out->flux.assign((nx + 1) * ny + nx * (ny + 1), 0.0);
    for (int64_t f = 0; f < nf; ++f) {
        const int64_t o = m.owner[f];
        const int64_t i = o % nx, j = o / nx;
        if (m.area[f].x != 0.0) {  // x-face: east face of the owner unless it is the inlet
            const bool west = m.area[f].x < 0.0;
            out->flux[(west ? i : i + 1) + (nx + 1) * j] = west ? -flux[f] : flux[f];
        } else {
            const bool south = m.area[f].y < 0.0;
            out->flux[(nx + 1) * ny + i + nx * (south ? j : j + 1)] = south ? -flux[f] : flux[f];
        }
    }
    return FLURSYS_OK;
}

// A face-based mesh handed in by a caller (the test meshes of the reference's
// own SIMPLE and momentum tests): cell centres and volumes, face owner,
// neighbour (-1 on the boundary), area vector and centre.
FvMesh mesh_from_arrays(int64_t nc, int64_t nf, const int64_t *owner, const int64_t *neigh, const double *area,
                        const double *fc, const double *cc, const double *vol) {
    FvMesh m;
    m.cc.resize(nc);
    m.vol.assign(vol, vol + nc);
    m.cell_faces.resize(nc);
    for (int64_t c = 0; c < nc; ++c) m.cc[c] = {cc[3 * c], cc[3 * c + 1], cc[3 * c + 2]};
    for (int64_t f = 0; f < nf; ++f) {
        m.owner.push_back(owner[f]);
        m.neigh.push_back(neigh[f]);
        m.area.push_back({area[3 * f], area[3 * f + 1], area[3 * f + 2]});
        m.fc.push_back({fc[3 * f], fc[3 * f + 1], fc[3 * f + 2]});
        m.patch.push_back(neigh[f] >= 0 ? kInternal : kBottom);
        m.cell_faces[owner[f]].push_back(f);
        if (neigh[f] >= 0) m.cell_faces[neigh[f]].push_back(f);
    }
    return m;
}

ScalarBc scalar_bc(int64_t nf, const int32_t *fixed, const double *value) {
    ScalarBc b;
    b.fixed.assign(nf, 0);
    b.value.assign(nf, 0.0);
    for (int64_t f = 0; f < nf; ++f) {
        b.fixed[f] = fixed ? fixed[f] : 0;
        b.value[f] = value ? value[f] : 0.0;
    }
    return b;
}

void export_csr(const OwnedCsr &P, int64_t *ro, int64_t *ci, double *v, int64_t cap, int64_t *nnz) {
    *nnz = (int64_t)P.v.size();
    if (ro) std::copy(P.ro.begin(), P.ro.end(), ro);
    for (int64_t k = 0; k < std::min<int64_t>(cap, *nnz); ++k) {
        if (ci) ci[k] = P.ci[k];
        if (v) v[k] = P.v[k];
    }
}

}  // namespace

// Face-based entry points (see flursys_oracle.h). Meshes are passed as
// (nc, nf, owner, neigh, area[3 nf], face centre[3 nf], cell centre[3 nc], volume[nc]).
#define ORC_MESH_ARGS int64_t nc, int64_t nf, const int64_t *owner, const int64_t *neigh, const double *area, \
                      const double *fc, const double *cc, const double *vol
#define ORC_MESH mesh_from_arrays(nc, nf, owner, neigh, area, fc, cc, vol)

extern "C" int32_t orc_fv_pressure_face_coefficients(ORC_MESH_ARGS, const double *rau, const int32_t *pc_fixed,
                                                     const double *pc_value, double *coef_out) {
    const FvMesh m = ORC_MESH;
    std::vector<double> r(rau, rau + nc), coef;
    const ScalarBc pcbc = scalar_bc(nf, pc_fixed, pc_value);
    const int32_t st = pressure_face_coefficients(m, r, pc_fixed ? &pcbc : nullptr, &coef);
    if (!st) std::copy(coef.begin(), coef.end(), coef_out);
    return st;
}

extern "C" int32_t orc_fv_correct_face_flux(ORC_MESH_ARGS, const double *predicted, const double *coef,
                                            const double *correction, const int32_t *pc_fixed,
                                            const double *pc_value, double *out) {
    const FvMesh m = ORC_MESH;
    const ScalarBc pcbc = scalar_bc(nf, pc_fixed, pc_value);
    std::vector<double> res;
    const int32_t st = correct_face_flux(m, std::vector<double>(predicted, predicted + nf),
                                         std::vector<double>(coef, coef + nf),
                                         std::vector<double>(correction, correction + nc),
                                         pc_fixed ? &pcbc : nullptr, &res);
    if (!st) std::copy(res.begin(), res.end(), out);
    return st;
}

extern "C" int32_t orc_fv_assemble_pressure_correction(ORC_MESH_ARGS, const double *predicted, const double *coef,
                                                       const int32_t *pc_fixed, const double *pc_value,
                                                       int64_t reference_cell, int64_t *ro, int64_t *ci, double *v,
                                                       int64_t cap, int64_t *nnz, double *rhs) {
    const FvMesh m = ORC_MESH;
    const ScalarBc pcbc = scalar_bc(nf, pc_fixed, pc_value);
    OwnedCsr P;
    std::vector<double> b;
    const int32_t st = assemble_pressure_correction(m, std::vector<double>(predicted, predicted + nf),
                                                    std::vector<double>(coef, coef + nf),
                                                    pc_fixed ? &pcbc : nullptr, reference_cell, &P, &b);
    if (st) return st;
    export_csr(P, ro, ci, v, cap, nnz);
    std::copy(b.begin(), b.end(), rhs);
    return FLURSYS_OK;
}

extern "C" int32_t orc_fv_continuity_rms(ORC_MESH_ARGS, const double *flux, double *out) {
    const FvMesh m = ORC_MESH;
    *out = continuity_rms(m, std::vector<double>(flux, flux + nf));
    return std::isfinite(*out) ? FLURSYS_OK : FLURSYS_ERR_INVALID_CONFIG;
}

extern "C" int32_t orc_fv_correct_cell_velocity(int64_t nc, const double *predictor, const double *rau,
                                                const double *grad, double *out) {
    std::vector<V3> pr(nc), g(nc), res;
    for (int64_t c = 0; c < nc; ++c) {
        pr[c] = {predictor[3 * c], predictor[3 * c + 1], predictor[3 * c + 2]};
        g[c] = {grad[3 * c], grad[3 * c + 1], grad[3 * c + 2]};
    }
    const int32_t st = correct_cell_velocity(pr, std::vector<double>(rau, rau + nc), g, &res);
    if (st) return st;
    for (int64_t c = 0; c < nc; ++c) {
        out[3 * c] = res[c].x;
        out[3 * c + 1] = res[c].y;
        out[3 * c + 2] = res[c].z;
    }
    return FLURSYS_OK;
}

extern "C" int32_t orc_fv_initial_face_flux(ORC_MESH_ARGS, const double *velocity, const double *wall_flux,
                                            double *out) {
    const FvMesh m = ORC_MESH;
    std::vector<V3> U(nc);
    for (int64_t c = 0; c < nc; ++c) U[c] = {velocity[3 * c], velocity[3 * c + 1], velocity[3 * c + 2]};
    const std::vector<double> f = initial_face_flux(m, U, std::vector<double>(wall_flux, wall_flux + nf));
    std::copy(f.begin(), f.end(), out);
    return FLURSYS_OK;
}

extern "C" int32_t orc_fv_assemble_momentum(ORC_MESH_ARGS, double nu, const int32_t *fixed, const double *value,
                                            const double *flux, const double *source, const double *current,
                                            double alpha, int64_t *ro, int64_t *ci, double *v, int64_t cap,
                                            int64_t *nnz, double *rhs) {
    const FvMesh m = ORC_MESH;
    const ScalarBc bc = scalar_bc(nf, fixed, value);
    OwnedCsr A;
    std::vector<double> b;
    const int32_t st = assemble_momentum(m, nu, bc, std::vector<double>(flux, flux + nf),
                                         source ? std::vector<double>(source, source + nc) : std::vector<double>(nc, 0.0),
                                         current ? std::vector<double>(current, current + nc) : std::vector<double>(nc, 0.0),
                                         alpha, &A, &b);
    if (st) return st;
    export_csr(A, ro, ci, v, cap, nnz);
    std::copy(b.begin(), b.end(), rhs);
    return FLURSYS_OK;
}

extern "C" int32_t orc_fv_simple(ORC_MESH_ARGS, const int32_t *vel_fixed, const double *vel_value,
                                 const int32_t *p_fixed, const double *p_value, const int32_t *pc_fixed,
                                 const double *pc_value, int64_t reference_cell, double nu,
                                 double velocity_relaxation, double pressure_relaxation, int64_t max_outer,
                                 double continuity_tolerance, const FlursysLinearSolverOptions *momentum_solver,
                                 const FlursysLinearSolverOptions *pressure_solver, double *velocity,
                                 double *pressure, double *face_flux, double *history, FlursysSimpleReport *report) {
    const FvMesh m = ORC_MESH;
    SimpleSetup su;
    for (int k = 0; k < 3; ++k) {
        su.vel[k] = scalar_bc(nf, vel_fixed, nullptr);
        for (int64_t f = 0; f < nf; ++f) su.vel[k].value[f] = vel_value[3 * f + k];
    }
    su.pbc = scalar_bc(nf, p_fixed, p_value);
    const ScalarBc pcbc = scalar_bc(nf, pc_fixed, pc_value);
    su.pcbc = pc_fixed ? &pcbc : nullptr;
    su.reference_cell = reference_cell;
    su.nu = nu;
    su.velocity_relaxation = velocity_relaxation;
    su.pressure_relaxation = pressure_relaxation;
    su.max_outer = max_outer;
    su.continuity_tolerance = continuity_tolerance;
    su.momentum_solver = *momentum_solver;
    su.pressure_solver = *pressure_solver;
    std::vector<V3> U(nc);
    for (int64_t c = 0; c < nc; ++c) U[c] = {velocity[3 * c], velocity[3 * c + 1], velocity[3 * c + 2]};
    std::vector<double> p(pressure, pressure + nc), flux(face_flux, face_flux + nf);
    SimpleOut out;
    const int32_t st = simple_solve(m, su, U, p, flux, &out);
    if (st) return st;
    for (int64_t c = 0; c < nc; ++c) {
        velocity[3 * c] = U[c].x;
        velocity[3 * c + 1] = U[c].y;
        velocity[3 * c + 2] = U[c].z;
    }
    std::copy(p.begin(), p.end(), pressure);
    std::copy(flux.begin(), flux.end(), face_flux);
    if (history) std::copy(out.history.begin(), out.history.end(), history);
    if (report) *report = out.rep;
    return FLURSYS_OK;
}

extern "C" int32_t orc_simple_channel(const FlursysSimpleConfig *cfg, double *velocity_x, double *velocity_y,
                                      double *pressure, double *face_flux, double *continuity_history,
                                      FlursysSimpleReport *report) {
    if (!cfg) return FLURSYS_ERR_INVALID_ARGUMENT;
    SimpleOut out;
    const int32_t st = simple_channel(*cfg, &out);
    if (st) return st;
    const size_t n = out.p.size();
    if (velocity_x) std::memcpy(velocity_x, out.u.data(), n * sizeof(double));
    if (velocity_y) std::memcpy(velocity_y, out.v.data(), n * sizeof(double));
    if (pressure) std::memcpy(pressure, out.p.data(), n * sizeof(double));
    if (face_flux) std::memcpy(face_flux, out.flux.data(), out.flux.size() * sizeof(double));
    if (continuity_history) std::memcpy(continuity_history, out.history.data(), out.history.size() * sizeof(double));
    if (report) *report = out.rep;
    return FLURSYS_OK;
}
