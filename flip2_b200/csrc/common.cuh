// common.cuh -- shared definitions of the sm_100a kernels: status handling,
// bounded look-back waits, warp/block reductions and the grid descriptor.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "flip2_b200.h"

namespace flip {

// Device error word bits (written with atomicOr, read by the host after a
// synchronisation point).
enum : uint32_t {
    DEVERR_LOOKBACK_TIMEOUT = 1u << 0,  // a decoupled look-back wait gave up
    DEVERR_TILE_OVERFLOW = 1u << 1,     // more particles in a tile than staged
    DEVERR_BAD_KEY = 1u << 2,           // a key outside the declared key range
    DEVERR_TMA_TIMEOUT = 1u << 3,       // a TMA copy's mbarrier wait gave up
};

// Upper bound on polls of a look-back status word before giving up.  The
// predecessor tile is always owned by a resident CTA (tiles are handed out in
// launch order through an atomic counter), so the wait normally ends within
// a few hundred polls; the bound only keeps a fault from hanging the GPU.
constexpr uint32_t kSpinLimit = 1u << 22;

#define FLIP_CUDA_TRY(expr)                                  \
    do {                                                     \
        cudaError_t _e = (expr);                             \
        if (_e != cudaSuccess) return ::flip::set_cuda_error(_e, #expr); \
    } while (0)

int set_cuda_error(cudaError_t e, const char* what);

// flip_sort_pairs with extra controls (sort.cu): err_accum, when not null,
// is a device word that receives the look-back timeout bit instead of the
// scratch's own error word; tile_base > 0 leaves the first tile_base tiles
// of every pass unclaimed (the timeout test only); head_dense, when not
// null, receives the segment heads of the sorted keys: head_dense[k] = the
// output index of the first key equal to k for every k < head_limit that
// occurs, 0xFFFFFFFF for the others (the last pass finds them as it
// scatters).
int sort_pairs_ex(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out, uint32_t* vals_out, uint64_t n,
                  int key_bits, void* scratch, size_t scratch_bytes, cudaStream_t s, uint32_t* err_accum,
                  uint32_t spin_limit, uint32_t tile_base, uint32_t* head_dense = nullptr, uint32_t head_limit = 0);
void set_error_text(const char* text);
const char* error_text();

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// ------------------------------------------------- dependent launches
// Programmatic dependent launch: a kernel launched with pdl_launch() may be
// scheduled while its predecessor on the stream is still finishing (its
// launch overlaps the predecessor's tail).  Such a kernel calls pdl_wait()
// before it touches global memory: the call returns once the predecessor
// has completed and its writes are visible.  In a kernel launched the
// ordinary way pdl_wait() returns at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t pdl_launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// --------------------------------------------------------------- device
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Inclusive warp scan of u32.
__device__ __forceinline__ uint32_t warp_inclusive_scan(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Exclusive scan of one u32 per thread over a block of NT threads; returns
// the exclusive prefix, writes the block total to *total.  Uses `sh` (NT/32
// words) and two __syncthreads.
template <int NT>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* sh, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = warp_inclusive_scan(v);
    if (lane == 31) sh[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = (lane < NT / 32) ? sh[lane] : 0u;
        uint32_t wi = warp_inclusive_scan(w);
        if (lane < NT / 32) sh[lane] = wi - w;
        if (lane == NT / 32 - 1) sh[NT / 32] = wi;
    }
    __syncthreads();
    uint32_t r = inc - v + sh[warp];
    *total = sh[NT / 32];
    return r;
}

// Deterministic FP64 block sum (fixed shuffle tree, fixed warp order).
template <int NT>
__device__ __forceinline__ double block_sum_f64(double v, double* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (warp == 0) {
        r = (lane < NT / 32) ? sh[lane] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;  // valid in thread 0
}

}  // namespace flip
