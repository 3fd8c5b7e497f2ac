// pcg3d_seq.cuh — host interface of the graph-driven 3D pressure PCG.
#pragma once

#include <cuda_runtime.h>

#include "pcg3d.cuh"

namespace flursys {

// Scalar state of one solve, read and written by the kernels of the graph.
struct CgSeqState {
    double rz_old, rz_new, alpha, beta;
    double residual, initial, initial_l2, threshold, true_l2;
    long long iterations;
    int first, done, status, error, replace, pending_conv;
    unsigned counter;  // last-block arrival counter
    unsigned device_error;  // DeviceError bits (a grid barrier of the resident solve gave up)
    // resident solve, as seen by block 0 (ns): [0] halo and direction update,
    // [1] operator pass, [2] grid barriers and reductions, [3] update and
    // residual replacements, [4] block 0's waits in grid barriers, [5] the
    // largest [0] + [1] + [3] of any block (the slowest block's work)
    unsigned long long phase_ns[6];
};

struct Pcg3dResPlan;

struct Pcg3dSeqPlan {
    Pcg3dResPlan *resident = nullptr;  // the chip-resident solve replaces the graph when it fits
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    double *partials = nullptr;
    CgSeqState *state = nullptr;
    int precision = 0;
    int host_iterations = 0;    // > 0: host-driven mode (diagnostics; FLURSYS_PCG_VARIANT=host)
    void *host_args = nullptr;  // argument block of the kernels
    void *cg1_maps = nullptr;   // tensor maps of the single-reduction step kernel
};

// Builds and instantiates the solve graph for fixed buffers (args as for
// pcg3d_launch, barrier/result/partials unused).
cudaError_t pcg3d_seq_plan(Pcg3dSeqPlan &plan, const Pcg3dArgs &args, int precision, int device);
cudaError_t pcg3d_seq_launch(const Pcg3dSeqPlan &plan, cudaStream_t stream);
void pcg3d_seq_destroy(Pcg3dSeqPlan &plan);
cudaError_t pcg3d_seq_run_host(const Pcg3dSeqPlan &plan, cudaStream_t stream);

}  // namespace flursys
