// cavity3d.cuh — host interface of the 3D velocity-phase kernels.
#pragma once

#include <cuda_runtime.h>

namespace flursys {

// Device pointers and constants of one 3D cavity; all arrays FP64.
struct Cavity3dState {
    int nx, ny, nz, sms;
    double dx, dy, dz, nu, lid, rho;
    double *u, *v, *w, *us, *vs, *ws, *p, *rhs;
};

// Reductions of the diagnostics pass. bad_index[f] is the first non-finite
// flat index of p, u, v, w (all ones when none).
struct Diag3Dev {
    double max_divergence;
    double max_speed;
    unsigned long long bad_index[4];
};

cudaError_t cavity3d_predict(const Cavity3dState &s, double dt, cudaStream_t st);
cudaError_t cavity3d_rhs(const Cavity3dState &s, double dt, cudaStream_t st);
cudaError_t cavity3d_correct(const Cavity3dState &s, double dt, cudaStream_t st);
cudaError_t cavity3d_diagnostics(const Cavity3dState &s, Diag3Dev *out, cudaStream_t st);

}  // namespace flursys
