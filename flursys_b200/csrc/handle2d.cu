// handle2d.cu — IncompressibleSolver (src/solver/incompressible.rs:294-746)
// on the device: case data, initial field, one advance_one_step and field
// access. Time-step control (adaptive dt, t_end, steady test) runs on the
// host from the reductions each step reads back, as in the reference.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "capi_internal.cuh"
#include "cavity2d.cuh"
#include "pcg2d.cuh"

namespace flursys {

namespace {

// Case data (src/cases/mod.rs:120-227) with SolverBoundaryOverrides
// (src/preprocess.rs:1370-1388).
struct HostCase {
    FlursysCaseParams c;
    FlursysBoundaryOverride ov[4];

    int case_kind(int side, double *outlet) const {
        *outlet = 0.0;
        switch (c.kind) {
            case FLURSYS_CASE_CAVITY: return kBkVelocity;
            case FLURSYS_CASE_CYLINDER:
                if (side == FLURSYS_SIDE_LEFT) return kBkVelocity;
                if (side == FLURSYS_SIDE_RIGHT) return kBkOutlet;
                return kBkSymmetry;
            default: return side == FLURSYS_SIDE_RIGHT ? kBkOutlet : kBkVelocity;
        }
    }
    int kind(int side, double *outlet = nullptr) const {
        double dummy;
        double *o = outlet ? outlet : &dummy;
        switch (ov[side].kind) {
            case FLURSYS_BOUNDARY_VELOCITY: *o = 0.0; return kBkVelocity;
            case FLURSYS_BOUNDARY_PRESSURE_OUTLET: *o = ov[side].pressure; return kBkOutlet;
            case FLURSYS_BOUNDARY_SYMMETRY: *o = 0.0; return kBkSymmetry;
            default: return case_kind(side, o);
        }
    }
    void case_velocity(int side, double y, double *u, double *v) const {
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
                    const double eta = std::clamp((y - c.step_height) / (c.height - c.step_height), 0.0, 1.0);
                    *u = 6.0 * c.reference_velocity * eta * (1.0 - eta);
                } else if (side == FLURSYS_SIDE_RIGHT) {
                    *u = c.reference_velocity;
                }
                return;
            default:
                if (side == FLURSYS_SIDE_LEFT) {
                    const double eta = std::clamp(y / c.height, 0.0, 1.0);
                    *u = 6.0 * c.reference_velocity * eta * (1.0 - eta);
                } else if (side == FLURSYS_SIDE_RIGHT) {
                    *u = c.reference_velocity;
                }
                return;
        }
    }
    void velocity(int side, double y, double *u, double *v) const {
        switch (ov[side].kind) {
            case FLURSYS_BOUNDARY_VELOCITY: *u = ov[side].u; *v = ov[side].v; return;
            case FLURSYS_BOUNDARY_PRESSURE_OUTLET:
            case FLURSYS_BOUNDARY_SYMMETRY: *u = 0.0; *v = 0.0; return;
            default: case_velocity(side, y, u, v);
        }
    }
    void initial_velocity(double x, double y, double *u, double *v) const {
        *u = 0.0;
        *v = 0.0;
        switch (c.kind) {
            case FLURSYS_CASE_CAVITY: return;
            case FLURSYS_CASE_CYLINDER: {
                const double rad = 0.5 * c.cylinder_diameter;
                if ((x - c.cylinder_xc) * (x - c.cylinder_xc) + (y - c.cylinder_yc) * (y - c.cylinder_yc) <= rad * rad)
                    return;
                const double xp = c.cylinder_xc + 1.5 * c.cylinder_diameter;
                const double yp = c.cylinder_yc + 0.25 * c.cylinder_diameter;
                const double s2 = c.cylinder_diameter * c.cylinder_diameter;
                const double ddx = x - xp, ddy = y - yp;
                const double psi = c.cylinder_perturbation * std::exp(-(ddx * ddx + ddy * ddy) / s2);
                *u = c.reference_velocity + (-2.0 * ddy / s2 * psi);
                *v = 2.0 * ddx / s2 * psi;
                return;
            }
            case FLURSYS_CASE_BACKWARD_STEP:
                if (x < c.step_x && y < c.step_height) return;
                if (y > c.step_height) {
                    const double eta = std::clamp((y - c.step_height) / (c.height - c.step_height), 0.0, 1.0);
                    *u = 6.0 * c.reference_velocity * eta * (1.0 - eta);
                } else {
                    *u = c.reference_velocity;
                }
                return;
            default: {
                const double eta = std::clamp(y / c.height, 0.0, 1.0);
                *u = 6.0 * c.reference_velocity * eta * (1.0 - eta);
                return;
            }
        }
    }
    bool is_solid(double x, double y) const {
        if (c.kind == FLURSYS_CASE_CYLINDER) {
            const double rad = 0.5 * c.cylinder_diameter;
            return (x - c.cylinder_xc) * (x - c.cylinder_xc) + (y - c.cylinder_yc) * (y - c.cylinder_yc) <= rad * rad;
        }
        if (c.kind == FLURSYS_CASE_BACKWARD_STEP) return x < c.step_x && y < c.step_height;
        return false;
    }
};

}  // namespace

struct Handle2D {
    Cavity2dState s{};
    double current_dt = 0.0;
    double outlet_p = 0.0;
    bool project = false;
    double last_max_u = 0.0, last_max_v = 0.0;  // max |u|, |v| of the current state
    std::vector<double *> allocs;
    uint8_t *flags = nullptr;
    Pcg2dInstance *inst_dev = nullptr;
    Pcg2dInstance inst{};
    bool cluster = false;  // the pressure solve runs as one thread-block cluster
    Diag2Dev *h_diag = nullptr;
    int nblocks = 0;
};

namespace {

double *dalloc(Handle2D *h2, size_t n, cudaError_t *e) {
    double *p = nullptr;
    if (*e == cudaSuccess) *e = cudaMalloc(&p, sizeof(double) * std::max<size_t>(n, 1));
    if (*e == cudaSuccess) {
        h2->allocs.push_back(p);
        *e = cudaMemset(p, 0, sizeof(double) * std::max<size_t>(n, 1));
    }
    return p;
}

// apply_velocity_boundaries on host arrays (initial field only).
void host_boundaries(const HostCase &hc, int nx, int ny, double dx, double dy, const std::vector<uint8_t> &solid,
                     std::vector<double> &u, std::vector<double> &v) {
    auto sol = [&](int i, int j) { return solid[i + nx * j] != 0; };
    auto uo = [&](int i, int j) {
        if (i == 0) return !sol(0, j);
        if (i == nx) return !sol(nx - 1, j);
        return !sol(i - 1, j) && !sol(i, j);
    };
    auto vo = [&](int i, int j) {
        if (j == 0) return !sol(i, 0);
        if (j == ny) return !sol(i, ny - 1);
        return !sol(i, j - 1) && !sol(i, j);
    };
    double a, b;
    for (int j = 0; j < ny; ++j) {
        const double y = (j + 0.5) * dy;
        int k = hc.kind(FLURSYS_SIDE_LEFT);
        if (k == kBkVelocity) { hc.velocity(FLURSYS_SIDE_LEFT, y, &a, &b); u[(nx + 1) * j] = a; }
        else if (k == kBkSymmetry) u[(nx + 1) * j] = 0.0;
        else u[(nx + 1) * j] = u[1 + (nx + 1) * j];
        k = hc.kind(FLURSYS_SIDE_RIGHT);
        if (k == kBkVelocity) { hc.velocity(FLURSYS_SIDE_RIGHT, y, &a, &b); u[nx + (nx + 1) * j] = a; }
        else if (k == kBkSymmetry) u[nx + (nx + 1) * j] = 0.0;
        else u[nx + (nx + 1) * j] = u[nx - 1 + (nx + 1) * j];
    }
    for (int i = 0; i < nx; ++i) {
        const double x = (i + 0.5) * dx;
        (void)x;
        int k = hc.kind(FLURSYS_SIDE_BOTTOM);
        if (k == kBkVelocity) { hc.velocity(FLURSYS_SIDE_BOTTOM, 0.0, &a, &b); v[i] = b; }
        else if (k == kBkSymmetry) v[i] = 0.0;
        else v[i] = v[i + nx];
        k = hc.kind(FLURSYS_SIDE_TOP);
        if (k == kBkVelocity) { hc.velocity(FLURSYS_SIDE_TOP, hc.c.height, &a, &b); v[i + nx * ny] = b; }
        else if (k == kBkSymmetry) v[i + nx * ny] = 0.0;
        else v[i + nx * ny] = v[i + nx * (ny - 1)];
    }
    for (int j = 0; j < ny; ++j)
        for (int i = 1; i < nx; ++i)
            if (!uo(i, j)) u[i + (nx + 1) * j] = 0.0;
    for (int j = 1; j < ny; ++j)
        for (int i = 0; i < nx; ++i)
            if (!vo(i, j)) v[i + nx * j] = 0.0;
}

// adaptive_time_step (incompressible.rs:2308-2336): the diffusion limit uses
// max(alpha, nu) when the energy equation is on.
int32_t adaptive_dt(double current, double mu, double mv, double dx, double dy, double nu,
                    const FlursysCudaConfig &c, double *out, std::string *err) {
    const double rate = mu / dx + mv / dy;
    const double cfl_dt = rate > 2.220446049250313e-16 ? c.target_cfl / rate : c.max_dt;
    const double inv = 1.0 / (dx * dx) + 1.0 / (dy * dy);
    const double eff = c.physics.energy_model == FLURSYS_ENERGY_CONSTANT_PROPERTIES
                           ? std::max(c.physics.thermal_diffusivity, nu) : nu;
    const double diff_dt = c.target_diffusion_number / (eff * inv);
    const double stable = std::min(std::min(c.max_dt, cfl_dt), diff_dt);
    if (stable < c.min_dt) {
        *err = "required stable time step " + rust_sci(stable, 3) + " is below configured min_dt " +
               rust_sci(c.min_dt, 3) + "; CFL constraint=" + rust_sci(cfl_dt, 3) + ", diffusion constraint=" +
               rust_sci(diff_dt, 3);
        return FLURSYS_ERR_INVALID_CONFIG;
    }
    *out = std::clamp(std::min(stable, current * c.max_growth_factor), c.min_dt, c.max_dt);
    return FLURSYS_OK;
}

bool reached_end_time(const FlursysCudaConfig &c, double time) {
    const double tol = 2.220446049250313e-16 * std::max(std::fabs(c.t_end), 1.0) * 16.0;
    return c.coupling == FLURSYS_COUPLING_PROJECTION && time >= c.t_end - tol;
}

}  // namespace

void build_case2d(const FlursysCudaConfig &c, Case2dHost *out) {
    HostCase hc{};
    hc.c = c.case_params;
    std::memcpy(hc.ov, c.overrides, sizeof hc.ov);
    const int nx = (int)c.nx, ny = (int)c.ny;
    const double dx = c.case_params.length / nx, dy = c.case_params.height / ny;
    Case2dHost &o = *out;
    for (int side = 0; side < 4; ++side) o.kind[side] = hc.kind(side);
    hc.kind(FLURSYS_SIDE_RIGHT, &o.outlet_p);
    o.project = o.kind[FLURSYS_SIDE_RIGHT] != kBkOutlet;  // pressure_reference_required (:1625-1632)

    // masks and boundary data
    std::vector<uint8_t> solid(nx * ny);
    o.flags.assign(nx * ny, 0);
    o.fluid = 0;
    o.ref_cell = -1;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) solid[i + nx * j] = hc.is_solid((i + 0.5) * dx, (j + 0.5) * dy) ? 1 : 0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            uint8_t f = solid[i + nx * j] ? kCellSolid : 0;
            if (i + 1 == nx && !solid[i + nx * j] && o.kind[FLURSYS_SIDE_RIGHT] == kBkOutlet) f |= kCellOutlet;
            o.flags[i + nx * j] = f;
            if (!(f & 3)) ++o.fluid;
            if (!solid[i + nx * j] && o.ref_cell < 0) o.ref_cell = i + nx * j;
        }
    std::vector<double> &bul = o.bnd[0], &bur = o.bnd[1], &bvb = o.bnd[2], &bvt = o.bnd[3];
    std::vector<double> &gub = o.bnd[4], &gut = o.bnd[5], &gvl = o.bnd[6], &gvr = o.bnd[7];
    bul.assign(ny, 0.0); bur.assign(ny, 0.0); bvb.assign(nx, 0.0); bvt.assign(nx, 0.0);
    gub.assign(nx + 1, 0.0); gut.assign(nx + 1, 0.0); gvl.assign(ny + 1, 0.0); gvr.assign(ny + 1, 0.0);
    double a, b;
    for (int j = 0; j < ny; ++j) {
        hc.velocity(FLURSYS_SIDE_LEFT, (j + 0.5) * dy, &a, &b); bul[j] = a;
        hc.velocity(FLURSYS_SIDE_RIGHT, (j + 0.5) * dy, &a, &b); bur[j] = a;
    }
    for (int i = 0; i < nx; ++i) {
        hc.velocity(FLURSYS_SIDE_BOTTOM, 0.0, &a, &b); bvb[i] = b;
        hc.velocity(FLURSYS_SIDE_TOP, hc.c.height, &a, &b); bvt[i] = b;
    }
    for (int i = 0; i <= nx; ++i) {
        hc.velocity(FLURSYS_SIDE_BOTTOM, 0.0, &a, &b); gub[i] = a;
        hc.velocity(FLURSYS_SIDE_TOP, hc.c.height, &a, &b); gut[i] = a;
    }
    for (int j = 0; j <= ny; ++j) {
        hc.velocity(FLURSYS_SIDE_LEFT, j * dy, &a, &b); gvl[j] = b;
        hc.velocity(FLURSYS_SIDE_RIGHT, j * dy, &a, &b); gvr[j] = b;
    }
    // initialize_velocity (:588-620)
    std::vector<double> &u = o.u, &v = o.v;
    u.assign((size_t)(nx + 1) * ny, 0.0);
    v.assign((size_t)nx * (ny + 1), 0.0);
    auto sol = [&](int i, int j) { return solid[i + nx * j] != 0; };
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i <= nx; ++i) {
            hc.initial_velocity(i * dx, (j + 0.5) * dy, &a, &b);
            const bool open = i == 0 ? !sol(0, j) : (i == nx ? !sol(nx - 1, j) : !sol(i - 1, j) && !sol(i, j));
            u[i + (nx + 1) * j] = open ? a : 0.0;
        }
    for (int j = 0; j <= ny; ++j)
        for (int i = 0; i < nx; ++i) {
            hc.initial_velocity((i + 0.5) * dx, j * dy, &a, &b);
            const bool open = j == 0 ? !sol(i, 0) : (j == ny ? !sol(i, ny - 1) : !sol(i, j - 1) && !sol(i, j));
            v[i + nx * j] = open ? b : 0.0;
        }
    host_boundaries(hc, nx, ny, dx, dy, solid, u, v);
    o.max_u = 0.0;
    o.max_v = 0.0;
    for (double x : u) o.max_u = std::max(o.max_u, std::fabs(x));
    for (double x : v) o.max_v = std::max(o.max_v, std::fabs(x));
}

int32_t init2d(FlursysCudaHandle *h) {
    const FlursysCudaConfig &c = h->cfg;
    auto *h2 = new Handle2D();
    h->h2 = h2;
    Cavity2dState &s = h2->s;
    Case2dHost cs;
    build_case2d(c, &cs);
    const int nx = (int)c.nx, ny = (int)c.ny;
    s.nx = nx; s.ny = ny; s.sms = h->sms;
    s.dx = c.case_params.length / nx;
    s.dy = c.case_params.height / ny;
    s.rho = c.case_params.density;
    s.nu = c.case_params.kinematic_viscosity;
    s.convection = c.convection;
    for (int side = 0; side < 4; ++side) s.kind[side] = cs.kind[side];
    h2->outlet_p = cs.outlet_p;
    h2->project = cs.project;
    h2->current_dt = c.dt;
    h2->last_max_u = cs.max_u;
    h2->last_max_v = cs.max_v;
    const std::vector<uint8_t> &flags = cs.flags;
    const std::vector<double> &u = cs.u, &v = cs.v;
    const long long fluid = cs.fluid;
    const int ref_cell = cs.ref_cell;

    cudaError_t e = cudaSuccess;
    const size_t nc = (size_t)nx * ny, nu = (size_t)(nx + 1) * ny, nv = (size_t)nx * (ny + 1);
    s.u = dalloc(h2, nu, &e); s.v = dalloc(h2, nv, &e);
    s.un = dalloc(h2, nu, &e); s.vn = dalloc(h2, nv, &e);
    s.us = dalloc(h2, nu, &e); s.vs = dalloc(h2, nv, &e);
    s.p = dalloc(h2, nc, &e); s.rhs = dalloc(h2, nc, &e); s.pold = dalloc(h2, nc, &e);
    s.uc = dalloc(h2, nc, &e); s.vc = dalloc(h2, nc, &e); s.speed = dalloc(h2, nc, &e); s.vort = dalloc(h2, nc, &e);
    double *bd[8];
    for (int k = 0; k < 8; ++k) {
        bd[k] = dalloc(h2, cs.bnd[k].size(), &e);
        if (e == cudaSuccess) e = cudaMemcpy(bd[k], cs.bnd[k].data(), cs.bnd[k].size() * sizeof(double), cudaMemcpyHostToDevice);
    }
    s.bu_left = bd[0]; s.bu_right = bd[1]; s.bv_bottom = bd[2]; s.bv_top = bd[3];
    s.gu_bottom = bd[4]; s.gu_top = bd[5]; s.gv_left = bd[6]; s.gv_right = bd[7];
    if (e == cudaSuccess) e = cudaMemcpy(s.u, u.data(), nu * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s.v, v.data(), nv * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&h2->flags, nc);
    if (e == cudaSuccess) e = cudaMemcpy(h2->flags, flags.data(), nc, cudaMemcpyHostToDevice);
    s.flags = h2->flags;
    s.cylinder = c.case_params.kind == FLURSYS_CASE_CYLINDER;
    s.cylinder_mu = c.case_params.cylinder_mu;
    s.post_blocks = cavity2d_post_blocks(nx, ny, h->sms);
    s.partials = dalloc(h2, (size_t)s.post_blocks * cavity2d_post_parts(), &e);
    // Energy equation (src/physics.rs, incompressible.rs:349-350,1441-1530):
    // temperature starts uniform at initial_temperature.
    const FlursysPhysicsSettings &ph = c.physics;
    if (ph.energy_model == FLURSYS_ENERGY_CONSTANT_PROPERTIES) {
        double *t0 = dalloc(h2, nc, &e);
        s.temp_next = dalloc(h2, nc, &e);
        const std::vector<double> init(nc, ph.initial_temperature);
        if (e == cudaSuccess) e = cudaMemcpy(t0, init.data(), nc * sizeof(double), cudaMemcpyHostToDevice);
        s.temp = t0;
        s.alpha = ph.thermal_diffusivity;
        s.tsource = ph.source_temperature_rate;
        for (int side = 0; side < 4; ++side) {
            s.tkind[side] = ph.thermal[side].kind;
            s.twall[side] = ph.thermal[side].temperature;
        }
        if (ph.buoyancy == FLURSYS_BUOYANCY_BOUSSINESQ) {
            s.buoyancy = 1;
            s.gbx = ph.gravity_x * ph.thermal_expansion;
            s.gby = ph.gravity_y * ph.thermal_expansion;
            s.tref = ph.reference_temperature;
        }
    }
    if (e == cudaSuccess) e = cudaMalloc(&s.diag, sizeof(Diag2Dev));
    if (e == cudaSuccess) e = cudaMallocHost(&h2->h_diag, sizeof(Diag2Dev));
    if (e == cudaSuccess) e = h->pcg.allocate((long long)nc, c.precision, h->device, 2);
    if (e == cudaSuccess) e = cudaMalloc(&h->pcg.r_z, (c.precision == FLURSYS_PRECISION_MIXED ? 4 : 8) * nc);
    if (e == cudaSuccess) e = cudaMalloc(&h2->inst_dev, sizeof(Pcg2dInstance));
    if (e != cudaSuccess) return set_cuda_error(&h->err, e, "allocating the 2D solver");
    // pressure system descriptor (one instance)
    Pcg2dInstance &in = h2->inst;
    in.nx = nx; in.ny = ny;
    in.idx2 = 1.0 / (s.dx * s.dx);
    in.idy2 = 1.0 / (s.dy * s.dy);
    in.flags = h2->flags;
    in.x = s.p;
    in.rhs = s.rhs;
    in.r = h->pcg.r; in.z = h->pcg.r_z; in.d0 = h->pcg.d0; in.d1 = h->pcg.d1; in.q = h->pcg.q;
    in.outlet_pressure = h2->outlet_p;
    in.project = h2->project ? 1 : 0;
    in.ref_cell = ref_cell;
    in.count_fluid = fluid;
    in.block0 = 0;
    // Small grids are latency bound: three grid barriers per iteration cost
    // more than the work, so the solve gets one block per 512 cells
    // (FLURSYS_2D_CELLS_PER_BLOCK overrides), at most the co-resident grid.
    long long per_block = 512;
    if (const char *env = std::getenv("FLURSYS_2D_CELLS_PER_BLOCK")) per_block = std::max(1LL, std::atoll(env));
    in.nblocks = (int)std::max(1LL, std::min<long long>(h->pcg.grid, ((long long)nc + per_block - 1) / per_block));
    // A small system without solid or outlet cells (at most 8 cells per
    // thread) runs as one thread-block cluster instead: the hardware cluster
    // barrier replaces the software grid barrier. FLURSYS_2D_CLUSTER=0 keeps
    // the grid path.
    {
        const char *cl_env = std::getenv("FLURSYS_2D_CLUSTER");
        const int maxc = pcg2d_max_cluster(c.precision);
        const long long threads = (long long)maxc * pcg2d_block_size();
        if (!(cl_env && std::strcmp(cl_env, "0") == 0) && fluid == (long long)nc && (long long)nc <= 8 * threads &&
            maxc <= h->pcg.grid) {
            h2->cluster = true;
            in.nblocks = (int)std::max(1LL, std::min<long long>(maxc, ((long long)nc + pcg2d_block_size() - 1) /
                                                                          pcg2d_block_size()));
        }
    }
    in.partials = h->pcg.partials;
    in.barrier = h->pcg.barrier;
    in.result = h->pcg.result;
    in.solver = c.pressure_solver == FLURSYS_PRESSURE_SOR ? FLURSYS_PRESSURE_SOR : FLURSYS_PRESSURE_PCG;
    in.stop_rule = c.stop_rule == FLURSYS_STOP_REL_L2 ? FLURSYS_STOP_REL_L2 : FLURSYS_STOP_ABS_INF;
    in.tol = c.pressure_tolerance;
    in.atol = c.pressure_atol;
    in.rtol = c.pressure_rtol;
    in.omega = c.pressure_omega;
    in.max_iters = c.pressure_max_iters;
    in.replace_every = c.residual_replacement_every > 0 ? c.residual_replacement_every : 50;
    e = cudaMemcpy(h2->inst_dev, &in, sizeof in, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return set_cuda_error(&h->err, e, "uploading the 2D pressure descriptor");
    return FLURSYS_OK;
}

void free2d(FlursysCudaHandle *h) {
    Handle2D *h2 = h->h2;
    if (!h2) return;
    for (double *p : h2->allocs) cudaFree(p);
    cudaFree(h2->flags);
    cudaFree(h2->s.diag);
    cudaFree(h2->inst_dev);
    if (h2->h_diag) cudaFreeHost(h2->h_diag);
    delete h2;
    h->h2 = nullptr;
}

// advance_one_step (:622-746) + advance() (:523-555)
int32_t step2d(FlursysCudaHandle *h, FlursysStepReport *rep) {
    const FlursysCudaConfig &c = h->cfg;
    Handle2D *h2 = h->h2;
    Cavity2dState &s = h2->s;
    cudaStream_t st = h->stream;
    if (reached_end_time(c, h->time)) {
        h->err = "projection simulation has already reached t_end";
        return FLURSYS_ERR_REACHED_END_TIME;
    }
    double step_dt = c.dt;
    if (c.adaptive) {
        int32_t stt = adaptive_dt(h2->current_dt, h2->last_max_u, h2->last_max_v, s.dx, s.dy, s.nu, c, &step_dt, &h->err);
        if (stt) return stt;
    }
    if (c.coupling == FLURSYS_COUPLING_PROJECTION) {
        step_dt = std::min(step_dt, c.t_end - h->time);
        if (step_dt <= 0.0) {
            h->err = "projection simulation has already reached t_end";
            return FLURSYS_ERR_REACHED_END_TIME;
        }
    }
    if (c.adaptive) h2->current_dt = step_dt;
    const bool simple = c.coupling == FLURSYS_COUPLING_SIMPLE;
    const double relax = simple ? c.velocity_relaxation : 1.0;
    const size_t nc = (size_t)s.nx * s.ny;
    cudaError_t e = cudaEventRecord(h->ev[0], st);
    if (e == cudaSuccess) e = cavity2d_predict(s, step_dt, simple ? 1 : 0, relax, st);
    if (e == cudaSuccess) e = cavity2d_boundaries(s, s.us, s.vs, st);
    if (simple) {
        if (e == cudaSuccess) e = cudaMemcpyAsync(s.pold, s.p, nc * sizeof(double), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(s.p, 0, nc * sizeof(double), st);
    }
    if (e == cudaSuccess) e = cavity2d_rhs(s, s.rho / (relax * step_dt), st);
    if (e == cudaSuccess) e = cudaEventRecord(h->ev[1], st);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->pcg.barrier, 0, sizeof(GridBarrier), st);
    if (e == cudaSuccess)
        e = h2->cluster ? pcg2d_launch_cluster(h2->inst_dev, h2->inst.nblocks, c.precision, st)
                        : pcg2d_launch(h2->inst_dev, 1, h2->inst.nblocks, c.precision, st);
    if (e == cudaSuccess) e = cudaEventRecord(h->ev[2], st);
    if (e == cudaSuccess) e = cavity2d_correct(s, relax * step_dt / s.rho, st);
    if (simple && e == cudaSuccess) e = cavity2d_simple_relax(s, c.pressure_relaxation, st);
    if (e == cudaSuccess) e = cavity2d_boundaries(s, s.un, s.vn, st);
    if (e == cudaSuccess) e = cavity2d_post(s, st);
    if (s.temp && e == cudaSuccess) e = cavity2d_temperature(s, step_dt, st);
    if (e == cudaSuccess) e = cudaEventRecord(h->ev[3], st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->pcg.h_result, h->pcg.result, sizeof(PcgResultDev), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h2->h_diag, s.diag, sizeof(Diag2Dev), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return set_cuda_error(&h->err, e, "2D step");
    const PcgResultDev &r = *h->pcg.h_result;
    int32_t status = pcg_result_status(r, &h->err);
    if (status) return status;
    std::swap(s.u, s.un);
    std::swap(s.v, s.vn);
    h->step += 1;
    if (c.coupling == FLURSYS_COUPLING_PROJECTION) h->time += step_dt;
    else h->time = h->step * c.dt;
    const Diag2Dev &d = *h2->h_diag;
    if (s.temp) {  // advance_temperature's runtime CFL check (:1449-1457)
        const double tcfl = step_dt * (d.max_abs_uc / s.dx + d.max_abs_vc / s.dy);
        if (tcfl > 1.0) {
            h->err = "explicit thermal advection is unstable at step " + std::to_string((long long)h->step) +
                     ": CFL=" + rust_sci(tcfl, 3) + " exceeds 1";
            return FLURSYS_ERR_INVALID_CONFIG;
        }
        std::swap(s.temp, s.temp_next);
    }
    // ensure_finite (:1707-1742): the first non-finite value of pressure, u,
    // v, speed, then temperature, read back for the message
    const char *names[5] = {"pressure", "u", "v", "speed", "temperature"};
    const double *fields[5] = {s.p, s.u, s.v, s.speed, s.temp};
    for (int f = 0; f < (s.temp ? 5 : 4); ++f)
        if (d.bad_index[f] != ~0ull) {
            h->err = nonfinite_message(names[f], d.bad_index[f], fields[f], h->step, true);
            return FLURSYS_ERR_NON_FINITE;
        }
    h2->last_max_u = d.max_abs_u;
    h2->last_max_v = d.max_abs_v;
    float ms_step = 0.f, ms_p = 0.f;
    cudaEventElapsedTime(&ms_step, h->ev[0], h->ev[3]);
    cudaEventElapsedTime(&ms_p, h->ev[1], h->ev[2]);
    std::memset(rep, 0, sizeof *rep);
    rep->iteration = h->step;
    rep->time = h->time;
    rep->time_step = step_dt;
    rep->continuity_residual = d.max_divergence;
    rep->pressure_residual = r.residual;
    rep->pressure_iterations = r.iterations;
    rep->momentum_residual = std::max(d.du, d.dv);
    rep->max_speed = d.max_speed;
    rep->momentum_cfl = step_dt * (d.max_abs_u / s.dx + d.max_abs_v / s.dy);
    rep->viscous_diffusion_number = s.nu * step_dt * (1.0 / (s.dx * s.dx) + 1.0 / (s.dy * s.dy));
    if (s.cylinder) {
        const FlursysCaseParams &cp = c.case_params;
        const double q = 0.5 * cp.density * cp.reference_velocity * cp.reference_velocity * cp.cylinder_diameter;
        if (q > 0.0) {
            rep->drag_coefficient = d.fx / q;
            rep->lift_coefficient = d.fy / q;
        }
    }
    rep->converged = c.case_params.kind != FLURSYS_CASE_CYLINDER && h->step >= c.minimum_steps &&
                     rep->momentum_residual < c.steady_tolerance &&
                     rep->continuity_residual < 10.0 * c.pressure_tolerance;
    rep->reached_end_time = reached_end_time(c, h->time);
    rep->pressure_initial_residual = r.initial;
    rep->pressure_true_relative_residual = r.initial_l2 > 0.0 ? r.true_l2 / r.initial_l2 : 0.0;
    rep->pressure_solve_ms = ms_p;
    rep->step_ms = ms_step;
    rep->pressure_status = r.status;
    return FLURSYS_OK;
}

bool field_ptr2d(FlursysCudaHandle *h, int32_t id, double **p, size_t *n) {
    Handle2D *h2 = h->h2;
    if (!h2) { *p = nullptr; *n = 0; return false; }
    const Cavity2dState &s = h2->s;
    const size_t nc = (size_t)s.nx * s.ny, nu = (size_t)(s.nx + 1) * s.ny, nv = (size_t)s.nx * (s.ny + 1);
    switch (id) {
        case FLURSYS_FIELD_U: *p = s.u; *n = nu; return true;
        case FLURSYS_FIELD_V: *p = s.v; *n = nv; return true;
        case FLURSYS_FIELD_PRESSURE: *p = s.p; *n = nc; return true;
        case FLURSYS_FIELD_RHS: *p = s.rhs; *n = nc; return true;
        case FLURSYS_FIELD_U_STAR: *p = s.us; *n = nu; return true;
        case FLURSYS_FIELD_V_STAR: *p = s.vs; *n = nv; return true;
        case FLURSYS_FIELD_SPEED: *p = s.speed; *n = nc; return true;
        case FLURSYS_FIELD_VORTICITY: *p = s.vort; *n = nc; return true;
        case FLURSYS_FIELD_U_CELL: *p = s.uc; *n = nc; return true;
        case FLURSYS_FIELD_V_CELL: *p = s.vc; *n = nc; return true;
        case FLURSYS_FIELD_TEMPERATURE:
            if (!s.temp) break;
            *p = s.temp; *n = nc; return true;
        default: break;
    }
    *p = nullptr; *n = 0;
    return false;
}

// An uploaded velocity field changes the inputs of the next adaptive dt.
void on_upload2d(FlursysCudaHandle *h, int32_t id) {
    Handle2D *h2 = h->h2;
    if (!h2 || (id != FLURSYS_FIELD_U && id != FLURSYS_FIELD_V)) return;
    double *p = nullptr;
    size_t n = 0;
    field_ptr2d(h, id, &p, &n);
    std::vector<double> tmp(n);
    if (cudaMemcpy(tmp.data(), p, n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) return;
    double m = 0.0;
    for (double x : tmp) m = std::max(m, std::fabs(x));
    if (id == FLURSYS_FIELD_U) h2->last_max_u = m;
    else h2->last_max_v = m;
}

// flursys_cuda_stencil_pcg with nz == 1: the cavity operator (no solids, no
// outlet) with zero-mean projections, src/linear stop rule.
int32_t stencil_pcg2d(int64_t nx, int64_t ny, double dx, double dy, const double *rhs, double *x_inout,
                      int32_t precision, const FlursysLinearSolverOptions *o, FlursysLinearSolveReport *report) {
    const size_t n = (size_t)nx * ny;
    if (n >= (1ull << 31)) return FLURSYS_ERR_INVALID_ARGUMENT;
    int device = 0;
    cudaGetDevice(&device);
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return FLURSYS_ERR_CUDA;
    PcgWorkspace ws;
    double *dxp = nullptr, *drhs = nullptr;
    uint8_t *flags = nullptr;
    Pcg2dInstance *idev = nullptr;
    std::string err;
    int32_t status = FLURSYS_OK;
    cudaError_t e = ws.allocate((long long)n, precision, device, 2);
    if (e == cudaSuccess) e = cudaMalloc(&ws.r_z, (precision == FLURSYS_PRECISION_MIXED ? 4 : 8) * n);
    if (e == cudaSuccess) e = cudaMalloc(&dxp, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&drhs, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&flags, n);
    if (e == cudaSuccess) e = cudaMemsetAsync(flags, 0, n, st);
    if (e == cudaSuccess) e = cudaMalloc(&idev, sizeof(Pcg2dInstance));
    if (e == cudaSuccess) e = cudaMemcpyAsync(dxp, x_inout, sizeof(double) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(drhs, rhs, sizeof(double) * n, cudaMemcpyHostToDevice, st);
    Pcg2dInstance in{};
    in.nx = (int)nx; in.ny = (int)ny;
    in.idx2 = 1.0 / (dx * dx); in.idy2 = 1.0 / (dy * dy);
    in.flags = flags; in.x = dxp; in.rhs = drhs;
    in.r = ws.r; in.z = ws.r_z; in.d0 = ws.d0; in.d1 = ws.d1; in.q = ws.q;
    in.project = 1; in.ref_cell = 0; in.count_fluid = (long long)n;
    in.block0 = 0; in.nblocks = ws.grid;
    in.partials = ws.partials; in.barrier = ws.barrier; in.result = ws.result;
    in.solver = FLURSYS_PRESSURE_PCG; in.stop_rule = FLURSYS_STOP_REL_L2;
    in.atol = o->absolute_tolerance; in.rtol = o->relative_tolerance;
    in.max_iters = o->max_iterations; in.replace_every = 50;
    if (e == cudaSuccess) e = cudaMemcpyAsync(idev, &in, sizeof in, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ws.barrier, 0, sizeof(GridBarrier), st);
    if (e == cudaSuccess) e = pcg2d_launch(idev, 1, ws.grid, precision, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ws.h_result, ws.result, sizeof(PcgResultDev), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(x_inout, dxp, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) status = set_cuda_error(&err, e, "2D stencil PCG");
    if (!status) status = pcg_result_status(*ws.h_result, &err);
    if (!status && report) {
        const PcgResultDev &r = *ws.h_result;
        report->status = r.status;
        report->reserved = 0;
        report->iterations = r.iterations;
        report->initial_residual = r.initial;
        report->final_residual = r.residual;
        report->relative_residual = r.initial == 0.0 ? 0.0 : r.residual / r.initial;
    }
    ws.free_all();
    cudaFree(dxp);
    cudaFree(drhs);
    cudaFree(flags);
    cudaFree(idev);
    cudaStreamDestroy(st);
    if (status) set_global_error(err);
    return status;
}

}  // namespace flursys
