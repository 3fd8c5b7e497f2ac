// sor.cuh — red-black SOR pressure solves (the GPU form of
// PressureSolverKind::Sor). Not iterate-identical to the reference's
// lexicographic sweeps; it converges to the same pinned/projected system.
#pragma once

#include <string>

#include "capi_internal.cuh"

namespace flursys {

// 3D: solve_pressure_poisson (src/solver/incompressible_3d.rs:293-332) with
// the stop test of pressure_residual (:476-502). Result in ws.result
// (iterations, residual).
int32_t run_sor3d(PcgWorkspace &ws, int nx, int ny, int nz, double dx, double dy, double dz, double *p,
                  const double *rhs, double omega, double tol, long long max_iters, cudaStream_t stream,
                  std::string *err);

}  // namespace flursys
