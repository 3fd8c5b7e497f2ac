// cavity2d.cuh — host interface of the 2D projection-step kernels
// (src/solver/incompressible.rs), FP64 throughout.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace flursys {

enum BoundaryKindDev : int { kBkVelocity = 0, kBkSymmetry = 1, kBkOutlet = 2 };

// Reductions of one post-step pass (filled by cavity2d_post).
struct Diag2Dev {
    double max_divergence;  // max_divergence (:1569-1582)
    double max_speed;       // speed.max_abs()
    double max_abs_u, max_abs_v;
    double du, dv;          // max_field_difference of u and v (:2287-2292)
    double fx, fy;          // cylinder force sums (:1634-1676)
    double max_abs_uc, max_abs_vc;    // u_cell / v_cell max_abs (thermal CFL, :1449-1451)
    unsigned long long bad_index[5];  // first non-finite index of p, u, v, speed, temperature
};

// Device pointers and constants of one 2D grid. Layout (Field2D,
// src/field.rs:31): x fastest; u is (nx+1) x ny, v is nx x (ny+1).
struct Cavity2dState {
    int nx, ny, sms;
    double dx, dy, rho, nu;
    int convection;  // FlursysConvection
    int kind[4];     // BoundaryKindDev per side (left, right, bottom, top)
    const uint8_t *flags;  // CellFlag bits per cell
    // Prescribed normal-face velocities on the four sides and the tangential
    // wall velocities used by the ghost values of the momentum stencil.
    const double *bu_left, *bu_right;   // ny
    const double *bv_bottom, *bv_top;   // nx
    const double *gu_bottom, *gu_top;   // nx+1
    const double *gv_left, *gv_right;   // ny+1
    double *u, *v, *un, *vn;            // state and next state
    double *us, *vs, *p, *rhs, *pold;
    double *uc, *vc, *speed, *vort;
    int cylinder;                       // compute force sums
    double cylinder_mu;
    // Energy equation and Boussinesq force (src/physics.rs); temp is null
    // when the energy model is off.
    double *temp;                       // cell temperature of the current state
    double *temp_next;                  // advance_temperature output
    int buoyancy;                       // add g * beta * (T_face - T_ref) in the predictor
    double gbx, gby, tref;              // gravity_x * beta, gravity_y * beta, T_ref
    double alpha, tsource;              // thermal diffusivity, source temperature rate
    int tkind[4];                       // FlursysThermalBoundaryKind per side
    double twall[4];                    // fixed wall temperatures per side
    double *partials;                   // post-pass partial reductions
    int post_blocks;
    Diag2Dev *diag;
};

cudaError_t cavity2d_predict(const Cavity2dState &s, double dt, int with_pressure, double relax, cudaStream_t st);
// apply_velocity_boundaries (:1981-2044) on (u, v); interior blocked faces are
// already zero in every producer.
cudaError_t cavity2d_boundaries(const Cavity2dState &s, double *u, double *v, cudaStream_t st);
cudaError_t cavity2d_rhs(const Cavity2dState &s, double rho_over_dt, cudaStream_t st);
cudaError_t cavity2d_correct(const Cavity2dState &s, double dt_over_rho, cudaStream_t st);
cudaError_t cavity2d_simple_relax(const Cavity2dState &s, double relax, cudaStream_t st);
// compute_cell_fields (:1381-1439) of (un, vn) plus every diagnostic of
// advance_one_step (:716-731) against the old state (u, v).
cudaError_t cavity2d_post(const Cavity2dState &s, cudaStream_t st);
// advance_temperature (:1441-1493) from temp into temp_next on the corrected
// velocities (un, vn); flags the first non-finite result in bad_index[4].
cudaError_t cavity2d_temperature(const Cavity2dState &s, double dt, cudaStream_t st);
int cavity2d_post_blocks(int nx, int ny, int sms);
int cavity2d_post_parts();  // partial sums per post-pass block

}  // namespace flursys
