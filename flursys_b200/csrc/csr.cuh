// csr.cuh — device CSR kernels behind the src/linear entry points.
#pragma once

#include <cuda_runtime.h>
