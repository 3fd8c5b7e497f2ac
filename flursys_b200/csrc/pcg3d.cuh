// pcg3d.cuh — host interface of the persistent 3D pressure PCG kernel.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "common.cuh"

namespace flursys {

// Written by block 0 at the end of a solve.
struct PcgResultDev {
    int error;        // FlursysStatus of a failure, 0 when none
    int status;       // FlursysLinearStatus
    long long iterations;
    double initial;   // initial residual in the stop-rule norm
    double residual;  // final residual in the stop-rule norm
    double true_l2;   // FP64 ||b - A x||_2 of the returned solution
    double initial_l2;
    unsigned device_error;  // DeviceError bits
    unsigned pad;
    // Nanoseconds block 0 spent in: [0] stencil passes, [1] pointwise passes,
    // [2] grid barriers + partial reductions, [3] residual replacements;
    // [4], [5] are used by the chip-resident solve only.
    unsigned long long phase_ns[6];
};

struct Pcg3dArgs {
    int nx, ny, nz;
    double ix2, iy2, iz2;
    double *x;          // pressure, FP64, updated in place
    const double *rhs;  // Poisson right-hand side; the system is A x = -rhs
    void *r, *d0, *d1, *q;  // FP64 (F64) or FP32 (MIXED) work vectors, n each
    float *dx;          // MIXED solution increment, n
    double *partials;   // grid * pcg3d_num_partials()
    GridBarrier *barrier;
    PcgResultDev *result;
    int stop_rule;      // FlursysStopRule
    double tol, atol, rtol;
    long long max_iters;
    int replace_every;
    int precision_vec_width;  // cells per vector in the pointwise pass (4 FP32, 2 FP64)
    const unsigned char *row_class;  // ny*nz bytes: 3*missing(j) + missing(k)
    // Set by pcg3d_launch: arrivals the grid barriers wait for beyond the
    // launched blocks (0 except under an injected barrier fault), and the
    // poll limit of each barrier wait.
    int barrier_extra;
    long long spin_limit;
};

// Poll limit of the barrier waits of a launch that runs under an injected
// barrier fault: the waits give up after a few milliseconds instead of
// about a second.
constexpr long long kInjectedFaultSpinLimit = 100'000LL;

// Arrivals to add to the grid barriers of the next persistent 3D PCG launch
// (0 when no fault is pending); reading it clears it.
int take_injected_barrier_fault();

size_t pcg3d_vector_bytes(int precision);
// Device table of 3*missing(j) + missing(k) for every row (j, k) of an
// nx x ny x nz grid (missing = number of absent neighbours on that axis).
cudaError_t pcg3d_make_row_class(int ny, int nz, unsigned char **out, cudaStream_t stream);
cudaError_t pcg3d_max_grid(int precision, int device, int *grid);
int pcg3d_block_size();
int pcg3d_num_partials();
cudaError_t pcg3d_launch(const Pcg3dArgs &args, int grid, int precision, cudaStream_t stream);

}  // namespace flursys
