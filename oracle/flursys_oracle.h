/*
 * flursys_oracle.h — TEST INFRASTRUCTURE ONLY.
 *
 * C API of the CPU FP64 oracle: a restatement of the FLURSYS reference
 * algorithms on the structured projection path (src/solver/incompressible.rs,
 * src/solver/incompressible_3d.rs) and of src/linear (CSR, Jacobi, CG, PCG,
 * BiCGSTAB). It is the checker of the CUDA backend in the tests and the timed
 * CPU baseline of bench.py. The product library never links it.
 *
 * The configuration and report types are the POD types of the public header
 * include/flursys_cuda.h, so the same config drives the oracle and the
 * device backend.
 */
#ifndef FLURSYS_ORACLE_H
#define FLURSYS_ORACLE_H

#include "flursys_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Worker threads used by loops that the reference runs on its Rayon pool.
 * 1 keeps every reduction serial and left-to-right. */
void orc_set_threads(int32_t threads);
int32_t orc_get_threads(void);

/* ---- src/linear ---- */
int32_t orc_csr_validate(int64_t nrows, int64_t ncols, int64_t nnz, const int64_t *row_offsets,
                         const int64_t *columns, const double *values, char *msg, size_t msg_size);
/* CsrBuilder::add over `nentries` triplets, then finalize(). Output arrays must
 * hold nrows+1 offsets and nentries columns/values; *nnz_out receives the count. */
int32_t orc_csr_build(int64_t nrows, int64_t ncols, int64_t nentries, const int64_t *rows,
                      const int64_t *cols, const double *vals, int64_t *row_offsets_out,
                      int64_t *columns_out, double *values_out, int64_t *nnz_out);
int32_t orc_csr_spmv(int64_t nrows, int64_t ncols, int64_t nnz, const int64_t *row_offsets,
                     const int64_t *columns, const double *values, const double *input,
                     double *output);
int32_t orc_jacobi_inverse_diagonal(int64_t n, int64_t nnz, const int64_t *row_offsets,
                                    const int64_t *columns, const double *values,
                                    double *inverse_diagonal, int64_t *bad_row);
/* method: 0 = cg, 1 = pcg (Jacobi), 2 = bicgstab. */
int32_t orc_csr_solve(int32_t method, int64_t n, int64_t nnz, const int64_t *row_offsets,
                      const int64_t *columns, const double *values, const double *rhs,
                      double *x_inout, const FlursysLinearSolverOptions *options,
                      FlursysLinearSolveReport *report);

/* ---- free functions of incompressible.rs with known-answer tests ---- */
void orc_momentum_stability_numbers(double dt, double nu, double dx, double dy, double max_abs_u,
                                    double max_abs_v, double *cfl, double *diffusion_number);
/* thermal_diffusivity < 0 means None. Returns FLURSYS_ERR_INVALID_CONFIG and
 * fills msg when the stable step is below min_dt. */
int32_t orc_adaptive_time_step(double current_dt, double max_abs_u, double max_abs_v, double dx,
                               double dy, double nu, double thermal_diffusivity, double min_dt,
                               double max_dt, double target_cfl, double target_diffusion_number,
                               double max_growth_factor, double *dt_out, char *msg,
                               size_t msg_size);

/* ---- structured solvers (2D IncompressibleSolver, 3D LidDrivenCavity3DSolver) ---- */
typedef struct OracleSolver OracleSolver;
int32_t orc_default_config(int32_t dimension, FlursysCudaConfig *cfg);
int32_t orc_create(const FlursysCudaConfig *cfg, OracleSolver **out, char *msg, size_t msg_size);
int32_t orc_step(OracleSolver *s, int64_t nsteps, FlursysStepReport *report);
size_t orc_field_size(const OracleSolver *s, int32_t field_id);
int32_t orc_get_field(const OracleSolver *s, int32_t field_id, double *out, size_t n);
int32_t orc_set_field(OracleSolver *s, int32_t field_id, const double *in, size_t n);
int32_t orc_last_error(const OracleSolver *s, char *buf, size_t size);
void orc_destroy(OracleSolver *s);

/* Individual phases of one step, for phase-level parity tests. */
int32_t orc_phase_predict(OracleSolver *s, double step_dt);
int32_t orc_phase_rhs(OracleSolver *s, double step_dt);
int32_t orc_phase_pressure(OracleSolver *s, double *residual, int64_t *iterations);
int32_t orc_phase_correct(OracleSolver *s, double step_dt);
/* Reference diagnostics of the current state. */
double orc_max_divergence(const OracleSolver *s);
double orc_pressure_residual(const OracleSolver *s); /* the reference SOR stop residual */
double orc_max_speed(const OracleSolver *s);

/* Matrix-free structured pressure PCG (same operator as the device entry
 * flursys_cuda_stencil_pcg), FP64, reference iteration order. */
int32_t orc_stencil_pcg(int64_t nx, int64_t ny, int64_t nz, double dx, double dy, double dz,
                        const double *rhs, double *x_inout,
                        const FlursysLinearSolverOptions *options,
                        FlursysLinearSolveReport *report);

/* Steady collocated SIMPLE channel (src/simple.rs:148-314 with the case
 * resolution of src/unstructured_incompressible.rs:106-212,368-482), FP64,
 * same outputs as flursys_cuda_simple_channel. */
int32_t orc_simple_channel(const FlursysSimpleConfig *cfg, double *velocity_x, double *velocity_y,
                           double *pressure, double *face_flux, double *continuity_history,
                           FlursysSimpleReport *report);

/* ---- The SIMPLE building blocks on a caller-supplied face-based mesh ----
 * (the reference's own unit-test meshes: two cells, closed cavities,
 * channels). A mesh is (nc, nf, owner[nf], neigh[nf] (-1 on the boundary),
 * area vector[3 nf], face centre[3 nf], cell centre[3 nc], volume[nc]).
 * Boundary conditions are per face: fixed (1) or zero gradient (0) with a
 * value; a NULL pc_fixed means no pressure-correction boundary (the
 * reference-cell form). CSR outputs hold nc+1 offsets and up to `cap`
 * entries, *nnz receives the count. */
#define ORC_FV_MESH int64_t nc, int64_t nf, const int64_t *owner, const int64_t *neigh, const double *area, \
                    const double *fc, const double *cc, const double *vol
/* pressure_face_coefficients[_with_boundary] (simple.rs:342-410) */
int32_t orc_fv_pressure_face_coefficients(ORC_FV_MESH, const double *rau, const int32_t *pc_fixed,
                                          const double *pc_value, double *coef_out);
/* correct_face_flux[_with_boundary] (simple.rs:412-496) */
int32_t orc_fv_correct_face_flux(ORC_FV_MESH, const double *predicted, const double *coef,
                                 const double *correction, const int32_t *pc_fixed, const double *pc_value,
                                 double *out);
/* assemble_pressure_correction[_with_boundary] (simple.rs:518-643) */
int32_t orc_fv_assemble_pressure_correction(ORC_FV_MESH, const double *predicted, const double *coef,
                                            const int32_t *pc_fixed, const double *pc_value,
                                            int64_t reference_cell, int64_t *ro, int64_t *ci, double *v,
                                            int64_t cap, int64_t *nnz, double *rhs);
/* continuity_rms (simple.rs:706-718) */
int32_t orc_fv_continuity_rms(ORC_FV_MESH, const double *flux, double *out);
/* correct_cell_velocity_from_gradient (simple.rs:673-704); vectors as xyz triples */
int32_t orc_fv_correct_cell_velocity(int64_t nc, const double *predictor, const double *rau, const double *grad,
                                     double *out);
/* initial_face_flux (simple.rs:724-755) */
int32_t orc_fv_initial_face_flux(ORC_FV_MESH, const double *velocity, const double *wall_flux, double *out);
/* assemble_momentum_component (momentum.rs:180-341), steady, upwind, two-point diffusion */
int32_t orc_fv_assemble_momentum(ORC_FV_MESH, double nu, const int32_t *fixed, const double *value,
                                 const double *flux, const double *source, const double *current, double alpha,
                                 int64_t *ro, int64_t *ci, double *v, int64_t cap, int64_t *nnz, double *rhs);
/* solve_simple (simple.rs:148-314); velocity (3 nc), pressure, face_flux
 * carry the initial state in and the result out; history holds up to
 * max_outer + 1 continuity values. */
int32_t orc_fv_simple(ORC_FV_MESH, const int32_t *vel_fixed, const double *vel_value, const int32_t *p_fixed,
                      const double *p_value, const int32_t *pc_fixed, const double *pc_value,
                      int64_t reference_cell, double nu, double velocity_relaxation, double pressure_relaxation,
                      int64_t max_outer, double continuity_tolerance,
                      const FlursysLinearSolverOptions *momentum_solver,
                      const FlursysLinearSolverOptions *pressure_solver, double *velocity, double *pressure,
                      double *face_flux, double *history, FlursysSimpleReport *report);

#ifdef __cplusplus
}
#endif

#endif
