// noalloc.cu — the 3D matrix-free pressure PCG without any allocation.
//
// flursys_cuda_stencil_pcg_noalloc runs the same persistent PCG kernel as
// flursys_cuda_stencil_pcg (pcg3d.cu) on caller-owned device buffers, with
// every work vector, the per-block partial sums, the grid barrier and the
// result record carved out of one file-scope device array. It never calls
// cudaMalloc, cudaFree or any routine that allocates, so it suits callers
// whose device memory is fully owned by their own pool, callers running under
// a hard memory cap that a mid-run cudaMalloc could break, and callers that
// cannot afford the device-wide synchronisation cudaFree implies.
//
// Limits and sharing rules (stated in include/flursys_cuda.h):
//   * at most kMaxCells = 2^18 cells (64^3); larger grids are rejected;
//   * the array (about 9.2 MB) stays resident on every device that loads the
//     library until the process exits;
//   * all calls share it and it keeps the last call's contents, so calls
//     that overlap on the GPU (two streams, two threads) race; the barrier
//     and the result record are cleared on every call, and a barrier that
//     gives up waiting marks the record, so a timed-out solve reports
//     FLURSYS_ERR_TIMEOUT rather than the cleared record;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <mutex>

#include "capi_internal.cuh"
#include "common.cuh"
#include "flursys_cuda.h"
#include "pcg3d.cuh"

namespace flursys {

namespace {

constexpr long long kMaxCells = 1LL << 18;
constexpr int kMaxBlocks = 1024;
constexpr int kMaxDevices = 64;

// Layout of the scratch array, in doubles.
constexpr long long kOffR = 0;
constexpr long long kOffD0 = kOffR + kMaxCells;
constexpr long long kOffD1 = kOffD0 + kMaxCells;
constexpr long long kOffQ = kOffD1 + kMaxCells;
constexpr long long kOffDx = kOffQ + kMaxCells;                // kMaxCells floats
constexpr long long kOffPartials = kOffDx + kMaxCells / 2;      // kMaxBlocks * partials per block
constexpr long long kOffBarrier = kOffPartials + (long long)kMaxBlocks * 8;
constexpr long long kOffResult = kOffBarrier + 2;               // GridBarrier is 16 bytes
constexpr long long kResultDoubles = (sizeof(PcgResultDev) + 7) / 8;
constexpr long long kOffRowClass = kOffResult + kResultDoubles;  // kMaxCells bytes
constexpr long long kTotalDoubles = kOffRowClass + kMaxCells / 8 + 1;

static __device__ __align__(256) double g_pcg_scratch[kTotalDoubles];

// Per-row boundary class 3*missing(j) + missing(k), written straight into the
// scratch array.
__global__ void row_class_kernel(int ny, int nz) {
    unsigned char *rc = reinterpret_cast<unsigned char *>(g_pcg_scratch + kOffRowClass);
    const int n = ny * nz;
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
        const int j = row % ny, k = row / ny;
        rc[row] = (unsigned char)(3 * ((j == 0) + (j == ny - 1)) + ((k == 0) + (k == nz - 1)));
    }
}

std::mutex g_mutex;
double *g_scratch_ptr[kMaxDevices] = {};

// Failures only: the message goes to flursys_cuda_global_error().
void set_err(const char *msg) { set_global_error(msg); }

// Device address of the scratch array on the current device (looked up once).
int32_t scratch_on_current_device(double **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        set_err("no usable current CUDA device");
        return FLURSYS_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_pcg_scratch);
        if (e != cudaSuccess || !p) {
            set_err("cudaGetSymbolAddress of the PCG scratch array failed");
            return FLURSYS_ERR_CUDA;
        }
        g_scratch_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_ptr[dev];
    return FLURSYS_OK;
}

}  // namespace

}  // namespace flursys

using namespace flursys;

extern "C" int32_t flursys_cuda_stencil_pcg_noalloc(int64_t nx, int64_t ny, int64_t nz, double dx, double dy,
                                                    double dz, const double *rhs_device, double *x_device,
                                                    int32_t precision, const FlursysLinearSolverOptions *options,
                                                    FlursysLinearSolveReport *report, void *stream) {
    if (!rhs_device || !x_device || !options) {
        set_err("null argument");
        return FLURSYS_ERR_INVALID_ARGUMENT;
    }
    if (precision != FLURSYS_PRECISION_F64 && precision != FLURSYS_PRECISION_MIXED) {
        set_err("unknown precision");
        return FLURSYS_ERR_INVALID_ARGUMENT;
    }
    if (nx < 1 || ny < 1 || nz < 2) {
        set_err("the allocation-free PCG solves the 3D pinned system: need nx, ny >= 1 and nz >= 2");
        return FLURSYS_ERR_INVALID_ARGUMENT;
    }
    if (nx > kMaxCells || ny > kMaxCells || nz > kMaxCells || nx * ny * nz > kMaxCells) {
        set_err("grid exceeds the allocation-free PCG limit of 262144 cells (64^3)");
        return FLURSYS_ERR_INVALID_ARGUMENT;
    }
    if ((reinterpret_cast<uintptr_t>(x_device) | reinterpret_cast<uintptr_t>(rhs_device)) % 16 != 0) {
        set_err("x_device and rhs_device must be 16-byte aligned");
        return FLURSYS_ERR_INVALID_ARGUMENT;
    }
    if (!(std::isfinite(options->absolute_tolerance) && options->absolute_tolerance >= 0.0 &&
          std::isfinite(options->relative_tolerance) && options->relative_tolerance >= 0.0)) {
        set_err("iterative solver breakdown: invalid solver tolerance");
        return FLURSYS_ERR_BREAKDOWN;
    }
    double *base = nullptr;
    int32_t st = scratch_on_current_device(&base);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0, maxgrid = 0;
    cudaGetDevice(&dev);
    cudaError_t e = pcg3d_max_grid(precision, dev, &maxgrid);
    if (e != cudaSuccess) {
        set_err("occupancy query failed");
        return FLURSYS_ERR_CUDA;
    }
    const long long n = nx * ny * nz;
    const int bs = pcg3d_block_size();
    long long want = (n + (long long)bs * 4 - 1) / ((long long)bs * 4);
    int grid = (int)std::max(1LL, std::min<long long>({(long long)maxgrid, want, (long long)kMaxBlocks}));

    Pcg3dArgs a{};
    a.nx = (int)nx; a.ny = (int)ny; a.nz = (int)nz;
    a.ix2 = 1.0 / (dx * dx); a.iy2 = 1.0 / (dy * dy); a.iz2 = 1.0 / (dz * dz);
    a.x = x_device;
    a.rhs = rhs_device;
    a.r = base + kOffR; a.d0 = base + kOffD0; a.d1 = base + kOffD1; a.q = base + kOffQ;
    a.dx = reinterpret_cast<float *>(base + kOffDx);
    a.partials = base + kOffPartials;
    a.barrier = reinterpret_cast<GridBarrier *>(base + kOffBarrier);
    a.result = reinterpret_cast<PcgResultDev *>(base + kOffResult);
    a.stop_rule = FLURSYS_STOP_REL_L2;
    a.tol = 0.0;
    a.atol = options->absolute_tolerance;
    a.rtol = options->relative_tolerance;
    a.max_iters = options->max_iterations;
    a.replace_every = 50;
    a.precision_vec_width = precision == FLURSYS_PRECISION_MIXED ? 4 : 2;
    a.row_class = reinterpret_cast<const unsigned char *>(base + kOffRowClass);

    row_class_kernel<<<(int)std::min<long long>(1024, (ny * nz + 255) / 256), 256, 0, s>>>((int)ny, (int)nz);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemsetAsync(a.barrier, 0, sizeof(GridBarrier), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.result, 0, sizeof(PcgResultDev), s);
    if (e == cudaSuccess) e = pcg3d_launch(a, grid, precision, s);
    PcgResultDev res{};
    if (e == cudaSuccess) e = cudaMemcpyAsync(&res, a.result, sizeof res, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_err(cudaGetErrorString(e));
        return FLURSYS_ERR_CUDA;
    }
    if (res.device_error & kDevErrBarrierTimeout) {
        set_err("pressure solver: a device grid barrier timed out");
        return FLURSYS_ERR_TIMEOUT;
    }
    if (res.error) {
        set_err(res.error == FLURSYS_ERR_BREAKDOWN ? "PCG pressure solver encountered a singular search direction"
                                                   : "PCG pressure solver produced a non-finite residual");
        return res.error;
    }
    if (report) {
        report->status = res.status;
        report->reserved = 0;
        report->iterations = res.iterations;
        report->initial_residual = res.initial;
        report->final_residual = res.residual;
        report->relative_residual = res.initial == 0.0 ? 0.0 : res.residual / res.initial;
    }
    return FLURSYS_OK;
}

