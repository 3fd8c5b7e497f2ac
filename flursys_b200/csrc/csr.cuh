// csr.cuh — device result record of the src/linear CSR solves.
#pragma once

#include <cuda_runtime.h>

namespace flursys {

struct CsrResultDev {
    int error;   // FlursysStatus of a failure, 0 when none
    int status;  // FlursysLinearStatus
    long long iterations;
    double initial;
    double final_residual;
    unsigned long long bad_row;  // first non-finite SpMV row (all ones when none)
    unsigned device_error;       // DeviceError bits
    unsigned pad;
};

}  // namespace flursys
