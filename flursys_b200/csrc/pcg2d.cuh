// pcg2d.cuh — host interface of the persistent 2D pressure solvers (PCG and
// red-black SOR), batched over independent instances.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "pcg3d.cuh"

namespace flursys {

enum CellFlag : uint8_t {
    kCellSolid = 1,   // Case::is_solid at the cell centre
    kCellOutlet = 2,  // pressure_outlet_cell (incompressible.rs:2066-2080)
};

// One pressure system of one 2D grid. A launch solves every instance with
// its own contiguous range of blocks, its own bounded barrier and its own
// reductions, so instances of different sizes converge independently.
struct Pcg2dInstance {
    int nx, ny;
    double idx2, idy2;
    const uint8_t *flags;  // nx*ny CellFlag bits
    double *x;             // pressure, FP64, in/out
    const double *rhs;     // Poisson right-hand side; the system is A x = -rhs on fluid rows
    void *r, *z, *d0, *d1, *q;  // work vectors (FP64 or FP32), nx*ny each
    double outlet_pressure;
    int project;                // zero-mean projection (no pressure outlet)
    int ref_cell;               // SOR: first fluid cell (find_reference_cell), -1 if none
    long long count_fluid;      // cells that the projection averages over
    int block0, nblocks;        // blocks of the launch that own this instance
    double *partials;           // nblocks * pcg2d_num_partials()
    GridBarrier *barrier;
    PcgResultDev *result;
    int solver;                 // FLURSYS_PRESSURE_PCG or FLURSYS_PRESSURE_SOR
    int stop_rule;              // FLURSYS_STOP_ABS_INF or FLURSYS_STOP_REL_L2
    double tol, atol, rtol, omega;
    long long max_iters;
    int replace_every;          // MIXED: FP64 residual replacement period
    int pad;
};

cudaError_t pcg2d_max_grid(int precision, int device, int *grid);
int pcg2d_block_size();
int pcg2d_num_partials();
// Launches one cooperative grid over all instances (device array `inst`).
cudaError_t pcg2d_launch(const Pcg2dInstance *inst_dev, int ninst, int total_blocks, int precision,
                         cudaStream_t stream);
// Largest thread-block cluster the 2D solver kernel can run as (16 where the
// device allows non-portable sizes, else 8).
int pcg2d_max_cluster(int precision);
// Launches one instance (device pointer) as a single cluster of `nblocks`
// blocks, its passes separated by the hardware cluster barrier.
cudaError_t pcg2d_launch_cluster(const Pcg2dInstance *inst_dev, int nblocks, int precision, cudaStream_t stream);

}  // namespace flursys
