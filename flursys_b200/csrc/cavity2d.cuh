// cavity2d.cuh — host interface of the 2D projection-step kernels.
#pragma once

#include <cuda_runtime.h>
