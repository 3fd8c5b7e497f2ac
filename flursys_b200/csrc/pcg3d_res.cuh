// pcg3d_res.cuh — host interface of the chip-resident 3D pressure PCG
// (pcg3d_res.cu): one cooperative launch per solve, MIXED precision, for
// grids whose 32 x 32 x tz tiles (tz <= 16) fit one per SM.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "common.cuh"
#include "pcg3d.cuh"
#include "pcg3d_seq.cuh"

namespace flursys {

struct ResArgs {
    int nx, ny, nz, nxy, n;
    int tz;             // planes per tile (<= 16)
    int ntx, nty, ntz;  // tiles per axis
    float wx, wy, wz;   // FP32 operator weights 1/h^2
    double ix2, iy2, iz2;
    float inv_diag_f[27];  // FP32 Jacobi weights by missing-neighbour class 9*mx + 3*my + mz
    double inv_diag[27];   // the same weights widened to FP64 (for r.z)
    double *x;             // FP64 pressure, updated in place
    const double *rhs;     // the system is A x = -rhs
    float *face0, *face1;  // n floats each: tile faces exchanged between tiles (alternating buffers)
    double *partials;      // 2 * grid * 4 partial sums
    GridBarrier *bar;
    int barrier_extra;     // arrivals beyond the grid (an injected barrier fault; 0 otherwise)
    long long spin_limit;  // poll limit of each barrier wait
    CgSeqState *st;
    int stop_rule;
    double tol, atol, rtol;
    long long max_iters;
    int replace_every;
};

struct Pcg3dResPlan {
    bool enabled = false;
    ResArgs args{};
    bool single = false;             // single-reduction form (L2 stop rule)
    const void *kernel = nullptr;    // the launched kernel
    int block = 512;                 // its threads per block
    bool col32 = false;              // dot products: every product in FP64, or FP32 column sums
    int grid = 0;
    size_t smem = 0;
    double *partials = nullptr;
    GridBarrier *barrier = nullptr;
};

// Sets up the resident solve for `args` (MIXED work vectors: args.r and
// args.q are the FP32 face-exchange buffers); false when the grid does not fit one tile per
// SM, the device cannot hold a tile, or FLURSYS_PCG_RESIDENT=0.
bool pcg3d_res_plan(Pcg3dResPlan &plan, const Pcg3dArgs &args, int device);
// One solve; the result is written to *state (CgSeqState fields error,
// status, iterations, initial, initial_l2, residual, true_l2, device_error).
cudaError_t pcg3d_res_launch(const Pcg3dResPlan &plan, CgSeqState *state, cudaStream_t stream);
void pcg3d_res_destroy(Pcg3dResPlan &plan);

}  // namespace flursys
