// handle2d.cu — IncompressibleSolver (src/solver/incompressible.rs) on the device.
#include "capi_internal.cuh"
#include "pcg2d.cuh"

namespace flursys {

struct Handle2D {};

cudaError_t pcg2d_max_grid(int, int, int *grid) { *grid = 1; return cudaSuccess; }
int pcg2d_block_size() { return 256; }
int pcg2d_num_partials() { return 8; }

int32_t init2d(FlursysCudaHandle *h) { h->err = "2D backend not built yet"; return FLURSYS_ERR_UNSUPPORTED; }
void free2d(FlursysCudaHandle *) {}
int32_t step2d(FlursysCudaHandle *h, FlursysStepReport *) { h->err = "2D backend not built yet"; return FLURSYS_ERR_UNSUPPORTED; }
bool field_ptr2d(FlursysCudaHandle *, int32_t, double **p, size_t *n) { *p = nullptr; *n = 0; return false; }
void on_upload2d(FlursysCudaHandle *, int32_t) {}
int32_t stencil_pcg2d(int64_t, int64_t, double, double, const double *, double *, int32_t,
                      const FlursysLinearSolverOptions *, FlursysLinearSolveReport *) { return FLURSYS_ERR_UNSUPPORTED; }

}  // namespace flursys
