// sor.cu — persistent red-black SOR for the 3D pinned pressure system.
//
// Each sweep updates the cells with (i+j+k) even, then the odd ones, with
// the SOR update of solve_pressure_poisson (src/solver/incompressible_3d.rs:
// 299-322): candidate = (sum of neighbours, a missing neighbour replaced by
// the centre value, minus rhs) / (2(ix2+iy2+iz2)); p += omega (candidate - p);
// p(0,0,0) = 0. After each sweep the reference stop residual
// max |Lap(p) - rhs| over cells other than (0,0,0) (:476-502) is reduced and
// tested against `tol`. Bounded grid barriers separate the colours.
#include <cuda_runtime.h>

#include "common.cuh"
#include "sor.cuh"

namespace flursys {

namespace {

constexpr int kBlock = 256;

struct G {
    int nx, ny, nz;
    long long nxy, n;
    double ix2, iy2, iz2;
};

__device__ __forceinline__ void decode(const G &g, long long c, int &i, int &j, int &k) {
    k = int(c / g.nxy);
    long long rem = c - (long long)k * g.nxy;
    j = int(rem / g.nx);
    i = int(rem - (long long)j * g.nx);
}

__device__ __forceinline__ double nbsum(const G &g, const double *p, long long c, int i, int j, int k,
                                        double pc) {
    const double e = (i + 1 < g.nx) ? __ldcg(p + c + 1) : pc;
    const double w = (i > 0) ? __ldcg(p + c - 1) : pc;
    const double n = (j + 1 < g.ny) ? __ldcg(p + c + g.nx) : pc;
    const double s = (j > 0) ? __ldcg(p + c - g.nx) : pc;
    const double f = (k + 1 < g.nz) ? __ldcg(p + c + g.nxy) : pc;
    const double b = (k > 0) ? __ldcg(p + c - g.nxy) : pc;
    return g.ix2 * (e + w) + g.iy2 * (n + s) + g.iz2 * (f + b);
}

__global__ void __launch_bounds__(kBlock) sor3d_kernel(int nx, int ny, int nz, double ix2, double iy2, double iz2,
                                                       double *p, const double *rhs, double omega, double tol,
                                                       long long max_iters, double *part, GridBarrier *bar,
                                                       PcgResultDev *res) {
    __shared__ double s_red[kBlock / 32];
    const G g{nx, ny, nz, (long long)nx * ny, (long long)nx * ny * nz, ix2, iy2, iz2};
    const double diag = 2.0 * (ix2 + iy2 + iz2);
    const long long stride = (long long)gridDim.x * kBlock;
    const long long tid0 = (long long)blockIdx.x * kBlock + threadIdx.x;
    double residual = INFINITY;
    long long its = 0;
    int error = 0;
    for (long long it = 0; it < max_iters; ++it) {
        its = it + 1;
        for (int color = 0; color < 2; ++color) {
            for (long long c = tid0; c < g.n; c += stride) {
                int i, j, k;
                decode(g, c, i, j, k);
                if (((i + j + k) & 1) != color) continue;
                if (c == 0) { p[0] = 0.0; continue; }
                const double pc = __ldcg(p + c);
                const double cand = (nbsum(g, p, c, i, j, k, pc) - __ldcg(rhs + c)) / diag;
                p[c] = pc + omega * (cand - pc);
            }
            if (!grid_sync_report(bar, gridDim.x, &res->device_error)) return;
        }
        double m = 0.0;
        for (long long c = tid0; c < g.n; c += stride) {
            if (c == 0) continue;
            int i, j, k;
            decode(g, c, i, j, k);
            const double pc = __ldcg(p + c);
            const double lap = nbsum(g, p, c, i, j, k, pc) - diag * pc;
            m = fmax(m, fabs(lap - __ldcg(rhs + c)));
        }
        const double bm = block_max<kBlock>(m, s_red);
        if (threadIdx.x == 0) part[blockIdx.x * 4 + (it & 1)] = bm;
        if (!grid_sync_report(bar, gridDim.x, &res->device_error)) return;
        double s = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += kBlock) s = fmax(s, __ldcg(&part[b * 4 + (it & 1)]));
        residual = block_max<kBlock>(s, s_red);
        if (!isfinite(residual)) { error = FLURSYS_ERR_NON_FINITE; break; }
        if (residual < tol) break;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        res->error = error;
        res->status = residual < tol ? FLURSYS_LINEAR_CONVERGED : FLURSYS_LINEAR_MAX_ITERATIONS;
        res->iterations = its;
        res->initial = 0.0;
        res->residual = residual;
        res->true_l2 = 0.0;
        res->initial_l2 = 0.0;
        res->device_error = bar->error;
    }
}

}  // namespace

int32_t run_sor3d(PcgWorkspace &ws, int nx, int ny, int nz, double dx, double dy, double dz, double *p,
                  const double *rhs, double omega, double tol, long long max_iters, cudaStream_t stream,
                  std::string *err) {
    int per_sm = 0, sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sor3d_kernel, kBlock, 0);
    int grid = ws.grid;
    if (grid > sms * per_sm) grid = sms * per_sm;
    double ix2 = 1.0 / (dx * dx), iy2 = 1.0 / (dy * dy), iz2 = 1.0 / (dz * dz);
    void *params[] = {&nx, &ny, &nz, &ix2, &iy2, &iz2, &p, &rhs, &omega, &tol, &max_iters, &ws.partials, &ws.barrier,
                      &ws.result};
    cudaError_t e = cudaMemsetAsync(ws.barrier, 0, sizeof(GridBarrier), stream);
    if (e == cudaSuccess)
        e = cudaLaunchCooperativeKernel((const void *)sor3d_kernel, dim3(grid), dim3(kBlock), params, 0, stream);
    if (e != cudaSuccess) return set_cuda_error(err, e, "sor3d launch");
    return FLURSYS_OK;
}

}  // namespace flursys
