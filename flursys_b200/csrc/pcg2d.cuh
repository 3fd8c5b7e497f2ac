// pcg2d.cuh — host interface of the persistent 2D pressure PCG kernel.
#pragma once

#include <cuda_runtime.h>

namespace flursys {

cudaError_t pcg2d_max_grid(int precision, int device, int *grid);
int pcg2d_block_size();
int pcg2d_num_partials();

}  // namespace flursys
