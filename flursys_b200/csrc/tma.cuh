// tma.cuh — tensor-memory-accelerator (TMA) tile loads into shared memory on
// sm_100a: tensor-map encoding on the host (driver entry point fetched
// through the runtime, so no libcuda link), and the device side —
// mbarrier set-up, expected-transaction arrival, cp.async.bulk.tensor
// 3D tile loads (no multicast) and a bounded completion wait.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>

namespace flursys {

// ---------------------------------------------------------------- host side

// cuTensorMapEncodeTiled of the installed driver, or nullptr.
inline PFN_cuTensorMapEncodeTiled_v12000 tma_encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// Tiled map of a dense nx x ny x nz FP32 array (x fastest), box bx x by x bz,
// zero fill outside the array. Needs nx % 4 == 0 (16-byte row stride) and a
// 16-byte aligned base. Returns false when the driver refuses.
inline bool tma_map_f32_3d(CUtensorMap *map, const float *base, int nx, int ny, int nz, unsigned bx, unsigned by,
                           unsigned bz) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = tma_encode_fn();
    if (!fn || nx % 4 != 0 || (reinterpret_cast<uintptr_t>(base) & 15u) != 0) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
    const cuuint64_t strides[2] = {(cuuint64_t)nx * 4, (cuuint64_t)nx * ny * 4};
    const cuuint32_t box[3] = {bx, by, bz};
    const cuuint32_t es[3] = {1, 1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tiled map of a dense BF16 activation tensor [nz][ny][nx][c] (channels
// fastest), box bc channels x bx x by x 1 plane, zero fill outside the
// tensor. Needs c % 8 == 0 and a 16-byte aligned base. Returns false when
// the driver refuses.
inline bool tma_map_bf16_cxyz(CUtensorMap *map, const void *base, int c, int nx, int ny, int nz, unsigned bc,
                              unsigned bx, unsigned by) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = tma_encode_fn();
    if (!fn || c % 8 != 0 || (reinterpret_cast<uintptr_t>(base) & 15u) != 0) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
    const cuuint64_t strides[3] = {(cuuint64_t)c * 2, (cuuint64_t)c * nx * 2, (cuuint64_t)c * nx * ny * 2};
    const cuuint32_t box[4] = {bc, bx, by, 1};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void *>(base), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// -------------------------------------------------------------- device side

__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for phase `parity` of the barrier, at most `limit` polls (each
// followed by a short sleep); false when the limit ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, long long limit) {
    for (long long i = 0; i < limit; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        __nanosleep(64);
    }
    return false;
}

// 3D tile load of the box at (x, y, z) into shared memory, completion
// signalled on `bar` (transaction bytes). x * 4 bytes must be a multiple of
// 16; the other coordinates may be negative or beyond the array (zero fill).
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// 4D tile load (c, x, y, z) of a tma_map_bf16_cxyz map, completion on `bar`.
// c * 2 bytes must be a multiple of 16; x, y, z may be negative or beyond
// the tensor (zero fill). The destination is 128-byte aligned.
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c, int x, int y, int z,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

}  // namespace flursys
