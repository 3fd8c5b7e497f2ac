// csr.cu — src/linear on the device.
#include "capi_internal.cuh"

extern "C" {
int32_t flursys_cuda_csr_cg(int64_t, int64_t, const int64_t *, const int64_t *, const double *, const double *,
                            double *, const FlursysLinearSolverOptions *, FlursysLinearSolveReport *) {
    return FLURSYS_ERR_UNSUPPORTED;
}
int32_t flursys_cuda_csr_pcg(int64_t, int64_t, const int64_t *, const int64_t *, const double *, const double *,
                             double *, const FlursysLinearSolverOptions *, FlursysLinearSolveReport *) {
    return FLURSYS_ERR_UNSUPPORTED;
}
int32_t flursys_cuda_csr_bicgstab(int64_t, int64_t, const int64_t *, const int64_t *, const double *, const double *,
                                  double *, const FlursysLinearSolverOptions *, FlursysLinearSolveReport *) {
    return FLURSYS_ERR_UNSUPPORTED;
}
int32_t flursys_cuda_csr_spmv(int64_t, int64_t, int64_t, const int64_t *, const int64_t *, const double *,
                              const double *, double *) {
    return FLURSYS_ERR_UNSUPPORTED;
}
}
