// common.cuh — device helpers shared by the flursys_cuda kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cuda/atomic>
#include <stdint.h>

#include "flursys_cuda.h"

namespace flursys {

constexpr int kWarp = 32;

// Device-side error bits reported through ErrorWord.
enum DeviceError : unsigned {
    kDevErrBarrierTimeout = 1u,  // a grid barrier gave up waiting
    kDevErrNonFinite = 2u,       // a NaN/Inf reached a checked value
};

// Upper bound on polls of one grid-barrier wait (each poll sleeps ~32 ns or
// more): about one second, far above any legitimate wait of a co-resident grid.
constexpr long long kBarrierSpinLimit = 30'000'000LL;

struct GridBarrier {
    unsigned count;
    unsigned generation;
    unsigned error;  // DeviceError bits
    unsigned pad;
};

// Sense-free generation barrier for a cooperative (co-resident) launch.
// Every wait is bounded: on timeout the error word is set and the caller is
// told to leave its loop. Returns false when the barrier failed.
__device__ __forceinline__ bool grid_sync(GridBarrier *bar, unsigned nblocks,
                                          long long spin_limit = kBarrierSpinLimit) {
    if (nblocks == 1u) {  // one block: a block barrier orders its global accesses
        __syncthreads();
        return true;
    }
    __syncthreads();
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> cnt(bar->count);
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> gen(bar->generation);
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> err(bar->error);
        int ok = 1;
        const unsigned my_gen = gen.load(cuda::memory_order_acquire);
        const unsigned arrived = cnt.fetch_add(1u, cuda::memory_order_acq_rel);
        if (arrived == nblocks - 1u) {
            cnt.store(0u, cuda::memory_order_relaxed);
            gen.fetch_add(1u, cuda::memory_order_release);
        } else {
            long long spins = 0;
            while (gen.load(cuda::memory_order_acquire) == my_gen) {
                if (err.load(cuda::memory_order_relaxed) != 0u || ++spins > spin_limit) {
                    err.fetch_or(kDevErrBarrierTimeout, cuda::memory_order_relaxed);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Barrier over the whole (cooperative) grid.
__device__ __forceinline__ bool grid_sync(GridBarrier *bar) { return grid_sync(bar, gridDim.x); }

// A barrier whose failure is also recorded in a word of the kernel's result
// record. Blocks leave the kernel at the first failed barrier, so the block
// that would write the final record never gets there; the timeout bit set
// here is what tells the host that the solve did not finish.
__device__ __forceinline__ bool grid_sync_report(GridBarrier *bar, unsigned nblocks, unsigned *report_word,
                                                 long long spin_limit = kBarrierSpinLimit) {
    if (grid_sync(bar, nblocks, spin_limit)) return true;
    if (threadIdx.x == 0) atomicOr(report_word, (unsigned)kDevErrBarrierTimeout);
    return false;
}

// Deterministic block sum of one double per thread (fixed shuffle tree).
template <int BLOCK>
__device__ __forceinline__ double block_sum(double v, double *smem /* >= BLOCK/32 */) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) smem[wid] = v;
    __syncthreads();
    double t = 0.0;
    if (wid == 0) {
        t = lane < BLOCK / 32 ? smem[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    }
    __syncthreads();
    if (threadIdx.x == 0) smem[0] = t;
    __syncthreads();
    t = smem[0];
    __syncthreads();
    return t;
}

// Block sums of N values per thread, and optionally (MAX) the block maximum
// of one more, with one set of barriers; each value takes the same shuffle
// tree and order as block_sum / block_max, so the results are bit-identical
// to separate calls. smem holds at least (N + MAX) * BLOCK / 32 doubles.
template <int BLOCK, int N, bool MAX>
__device__ __forceinline__ void block_reduce_n(double (&v)[N], double &mx, double *smem) {
    constexpr int NW = BLOCK / 32;
#pragma unroll
    for (int k = 0; k < N; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if (MAX)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < N; ++k) smem[k * NW + wid] = v[k];
        if (MAX) smem[N * NW + wid] = mx;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            double t = lane < NW ? smem[k * NW + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            v[k] = t;
        }
        if (MAX) {
            double t = lane < NW ? smem[N * NW + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_xor_sync(0xffffffffu, t, o));
            mx = t;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < N; ++k) smem[k] = v[k];
        if (MAX) smem[N] = mx;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = smem[k];
    if (MAX) mx = smem[N];
    __syncthreads();
}
template <int BLOCK, int N>
__device__ __forceinline__ void block_sum_n(double (&v)[N], double *smem) {
    double unused = 0.0;
    block_reduce_n<BLOCK, N, false>(v, unused, smem);
}

template <int BLOCK>
__device__ __forceinline__ double block_max(double v, double *smem) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) smem[wid] = v;
    __syncthreads();
    double t = 0.0;
    if (wid == 0) {
        t = lane < BLOCK / 32 ? smem[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_xor_sync(0xffffffffu, t, o));
    }
    __syncthreads();
    if (threadIdx.x == 0) smem[0] = t;
    __syncthreads();
    t = smem[0];
    __syncthreads();
    return t;
}

// Sums NV interleaved partial sums (partials[b*NV + v], b < nblocks) in a
// fixed order; every calling block obtains bit-identical results.
template <int BLOCK, int NV>
__device__ __forceinline__ void reduce_partials(const double *__restrict__ partials, int nblocks,
                                                double *out, double *smem) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += BLOCK) s += __ldcg(&partials[b * NV + v]);
        out[v] = block_sum<BLOCK>(s, smem);
    }
}

template <int BLOCK, int NV>
__device__ __forceinline__ void reduce_partials_max(const double *__restrict__ partials,
                                                    int nblocks, double *out, double *smem) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += BLOCK) s = fmax(s, __ldcg(&partials[b * NV + v]));
        out[v] = block_max<BLOCK>(s, smem);
    }
}

}  // namespace flursys
