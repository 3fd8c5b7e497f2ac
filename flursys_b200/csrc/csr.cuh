// csr.cuh — device result record of the src/linear CSR solves.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "common.cuh"
#include "flursys_cuda.h"

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

// Work vectors of device-resident CSR solves (grown on demand), for callers
// inside the library that assemble their matrices on the device.
struct CsrDeviceWork {
    int n = 0, grid = 0;
    double *vec = nullptr;       // 10 vectors of n
    double *partials = nullptr;  // grid * 4
    double *inv_diag = nullptr;  // n (PCG)
    GridBarrier *bar = nullptr;
    CsrResultDev *res = nullptr;   // [0] the solve, [1] the Jacobi set-up (error only)
    CsrResultDev *hres = nullptr;  // pinned copy of both
    cudaError_t ensure(int n, int device);
    void release();
};

// Enqueues one solve on device-resident CSR arrays (32-bit indices, columns
// ascending in each row): method 0 CG, 1 Jacobi-PCG (the inverse diagonal is
// formed on the device; a missing or zero diagonal is reported as an error),
// 2 BiCGSTAB, with the stop rule of src/linear. The result record lands in
// w.hres after the stream is synchronised; csr_device_status maps it.
// (b and x are not checked for finiteness beforehand: a non-finite value
// surfaces as FLURSYS_ERR_NON_FINITE from the first SpMV or dot.)
cudaError_t csr_device_launch(int method, int n, const int *ro, const int *ci, const double *va, const double *b,
                              double *x, double atol, double rtol, long long max_iters, CsrDeviceWork &w,
                              cudaStream_t st);
int32_t csr_device_status(const CsrResultDev *hres, FlursysLinearSolveReport *rep, std::string *err);

}  // namespace flursys
