// tma.cuh -- tensor-memory-accelerator (TMA) staging for sm_100a kernels:
// mbarrier helpers with bounded waits, the 3-D tiled bulk-tensor load, and
// the host-side encoding of a 3-D FP32 tensor map.
//
// Only plain loads of this GPU's own buffers are issued here: no cluster
// multicast form of cp.async.bulk.tensor exists in this library.  Every
// tensor map's innermost box extent is a multiple of 16 bytes, and callers
// start every box at an x coordinate that is a multiple of 4 floats (16 B).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace flip {

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    // make the initialised barrier visible to the async (TMA) proxy
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// arrive on the barrier and expect `bytes` of transactions in this phase
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(smem_addr(bar)),
        "r"(bytes)
        : "memory");
}

__device__ __forceinline__ bool mbar_test_parity(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the barrier phase of the given parity to complete, polling at
// most `limit` times; false when the wait gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t it = 0; it < limit; ++it)
        if (mbar_test_parity(bar, parity)) return true;
    return false;
}

// order this thread's earlier generic-proxy accesses of shared memory before
// later async-proxy (TMA) accesses of it
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 3-D tiled load of one box of `map` at element coordinates (x, y, z) into
// shared memory at dst (128-byte aligned), completing on `bar`.
// Coordinates outside the tensor read as zero.  x must be a multiple of 4.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

// Host: encode the tensor map of a dense x-fastest FP32 grid of nx*ny*nz
// elements at `base` (256-byte aligned), with boxes of bx*by*bz elements
// (bx*4 a multiple of 16), out-of-range elements reading as zero.
int encode_grid_map_f32(CUtensorMap* map, const float* base, int nx, int ny, int nz, int bx, int by, int bz);

}  // namespace flip
