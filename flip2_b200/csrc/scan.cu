// scan.cu -- single-pass prefix sums with decoupled look-back (sm_100a).
//
//  * flip_inclusive_scan_u32 replaces cudaParallelPrefixSum
//    (engine/algorithms/parallelPrefixSumKernels.cu:5-77), a recursive
//    three-kernel Blelloch scan that allocates and frees its block sums on
//    every call.  One kernel, one read and one write per element.
//  * flip_segment_heads fuses markUniqueGridCells, the inclusive scan of the
//    head flags and mapNodeIndicesToParticles
//    (engine/algorithms/particleToGridFunctions.cu:303-345) into one pass
//    over the sorted keys, and leaves the segment count on the device.
//
// Tiles of 4096 elements are claimed in launch order through an atomic
// counter; each publishes (flag, value) in one 64-bit word, so a waiting CTA
// only ever waits on a resident predecessor.  Waits are bounded.
#include <mutex>
#include <string>
#include "common.cuh"

namespace flip {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr unsigned long long kStAgg = 1ull << 62;
constexpr unsigned long long kStPrefix = 2ull << 62;
constexpr unsigned long long kStFlags = 3ull << 62;

static inline size_t align_up_s(size_t v, size_t a) { return (v + a - 1) / a * a; }

struct ScanLayout {
    size_t err, ctr, status, total;
};
static ScanLayout scan_layout(uint64_t n) {
    ScanLayout L;
    uint64_t tiles = (n + kScanTile - 1) / kScanTile;
    size_t o = 0;
    L.err = o; o += 16;
    L.ctr = o; o = align_up_s(o + 16, 256);
    L.status = o; o = align_up_s(o + sizeof(unsigned long long) * (tiles ? tiles : 1), 256);
    L.total = o;
    return L;
}

__device__ __forceinline__ int pad_idx(int j) { return j + (j >> 5); }

// Decoupled look-back by one warp: publishes the tile's aggregate, then lane
// l reads predecessor tile - 1 - l of a 32-tile window; the window is summed
// once every tile up to the nearest inclusive prefix has published, and
// slides back 32 tiles while it holds none.  Publishes and returns the tile's
// exclusive prefix (u32, wrapping) on every lane.  A window reload counts as
// one poll against spin_limit.
__device__ __forceinline__ uint32_t lookback_warp_u32(unsigned long long* status, uint32_t tile, uint32_t agg,
                                                      uint32_t* err, uint32_t spin_limit) {
    const int lane = threadIdx.x & 31;
    if (tile == 0) {
        if (lane == 0) st_relaxed_u64(status, kStPrefix | agg);
        return 0u;
    }
    if (lane == 0) st_relaxed_u64(status + tile, kStAgg | agg);
    uint32_t excl = 0, spins = 0;
    bool timed_out = false;
    int64_t end = (int64_t)tile - 1;
    while (true) {
        const int64_t t = end - lane;
        const unsigned long long s = t >= 0 ? ld_relaxed_u64(status + t) : kStPrefix;
        const unsigned long long f = s & kStFlags;
        const uint32_t pre = __ballot_sync(0xffffffffu, f == kStPrefix);
        const uint32_t unset = __ballot_sync(0xffffffffu, f == 0ull);
        const int first = pre ? __ffs(pre) - 1 : 31;  // lanes 0 .. first are summed
        const uint32_t need = first >= 31 ? 0xffffffffu : ((2u << first) - 1u);
        if (unset & need) {
            if (++spins > spin_limit) {
                timed_out = true;
                break;
            }
            continue;
        }
        excl += warp_sum<uint32_t>(lane <= first ? (uint32_t)s : 0u);
        if (pre) break;
        end -= 32;
    }
    if (lane == 0) {
        if (timed_out) atomicOr(err, DEVERR_LOOKBACK_TIMEOUT);
        st_relaxed_u64(status + tile, kStPrefix | (uint32_t)(excl + agg));
    }
    return excl;
}

template <int MODE>  // 0: plain scan of `in`;  1: segment heads of sorted keys in `in`
__global__ void __launch_bounds__(kScanThreads) scan_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                            uint64_t n, unsigned long long* __restrict__ status,
                                                            uint32_t* __restrict__ ctr, uint32_t* __restrict__ err,
                                                            uint32_t* __restrict__ starts, uint32_t* __restrict__ node_keys,
                                                            uint32_t* __restrict__ d_count, uint32_t spin_limit,
                                                            uint32_t tile_base) {
    __shared__ uint32_t s_data[kScanTile + kScanTile / 32];
    __shared__ uint32_t s_prev_key;
    __shared__ uint32_t s_tile, s_excl;
    __shared__ uint32_t s_scan[kScanThreads / 32 + 1];
    const int tid = threadIdx.x;
    if (tid == 0) s_tile = atomicAdd(ctr, 1u) + tile_base;
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * kScanTile;
    if (MODE == 1 && tid == 0) s_prev_key = (base > 0) ? in[base - 1] : 0u;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        int j = i * kScanThreads + tid;
        uint64_t g = base + j;
        s_data[pad_idx(j)] = (g < n) ? in[g] : 0u;
    }
    __syncthreads();
    uint32_t v[kScanItems];
    uint32_t sum = 0;
    const int j0 = tid * kScanItems;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        uint32_t x;
        if (MODE == 0) {
            x = s_data[pad_idx(j0 + i)];
        } else {
            uint64_t g = base + j0 + i;
            uint32_t k = s_data[pad_idx(j0 + i)];
            uint32_t kp = (j0 + i == 0) ? s_prev_key : s_data[pad_idx(j0 + i - 1)];
            x = (g < n) && (g == 0 || k != kp) ? 1u : 0u;
        }
        sum += x;
        v[i] = sum;  // thread-local inclusive
    }
    uint32_t agg;
    uint32_t texcl = block_exclusive_scan<kScanThreads>(sum, s_scan, &agg);
    if (tid < 32) {
        const uint32_t e = lookback_warp_u32(status, tile, agg, err, spin_limit);
        if (tid == 0) s_excl = e;
    }
    __syncthreads();
    const uint32_t pre = s_excl + texcl;
    if (MODE == 0) {
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) s_data[pad_idx(j0 + i)] = pre + v[i];
        __syncthreads();
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) {
            int j = i * kScanThreads + tid;
            uint64_t g = base + j;
            if (g < n) out[g] = s_data[pad_idx(j)];
        }
    } else {
        // heads: write starts/keys from the thread-blocked view, then the scan
        uint32_t prevv = pre;
        uint32_t keys_local[kScanItems];
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) keys_local[i] = s_data[pad_idx(j0 + i)];
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) {
            uint64_t g = base + j0 + i;
            uint32_t sc = pre + v[i];
            if (g < n && sc != prevv) {
                starts[sc - 1] = (uint32_t)g;
                if (node_keys) node_keys[sc - 1] = keys_local[i];
            }
            if (g == n - 1) *d_count = sc;
            prevv = sc;
        }
        if (out) {
            __syncthreads();
#pragma unroll
            for (int i = 0; i < kScanItems; ++i) s_data[pad_idx(j0 + i)] = pre + v[i];
            __syncthreads();
#pragma unroll
            for (int i = 0; i < kScanItems; ++i) {
                int j = i * kScanThreads + tid;
                uint64_t g = base + j;
                if (g < n) out[g] = s_data[pad_idx(j)];
            }
        }
    }
}

// err_accum: a device word that the look-back timeout bit is OR-ed into
// instead of the scratch's own error word (an engine's persistent word);
// tile_base > 0 leaves the first tile_base tiles unclaimed, so that the
// look-back of tile tile_base waits on a status word nothing publishes (the
// timeout test of flip_test_lookback_timeout)
int launch_scan(int mode, const uint32_t* in, uint32_t* out, uint64_t n, void* scratch, size_t bytes, cudaStream_t s,
                uint32_t* starts, uint32_t* node_keys, uint32_t* d_count, uint32_t* err_accum, uint32_t spin_limit,
                uint32_t tile_base) {
    ScanLayout L = scan_layout(n);
    if (!scratch || bytes < L.total) {
        set_error_text("scan: scratch too small");
        return FLIP_ERR_ARG;
    }
    char* S = (char*)scratch;
    uint64_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tile_base >= tiles) {
        set_error_text("scan: tile_base beyond the tile count");
        return FLIP_ERR_ARG;
    }
    FLIP_CUDA_TRY(cudaMemsetAsync(S, 0, L.status + sizeof(unsigned long long) * tiles, s));
    uint32_t* err = err_accum ? err_accum : (uint32_t*)(S + L.err);
    uint32_t* ctr = (uint32_t*)(S + L.ctr);
    unsigned long long* st = (unsigned long long*)(S + L.status);
    const unsigned grid = (unsigned)(tiles - tile_base);
    if (mode == 0)
        scan_kernel<0><<<grid, kScanThreads, 0, s>>>(in, out, n, st, ctr, err, nullptr, nullptr, nullptr, spin_limit,
                                                     tile_base);
    else
        scan_kernel<1><<<grid, kScanThreads, 0, s>>>(in, out, n, st, ctr, err, starts, node_keys, d_count, spin_limit,
                                                     tile_base);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

size_t scan_scratch_bytes(uint64_t n) { return scan_layout(n).total; }

}  // namespace flip

using namespace flip;

extern "C" size_t flip_inclusive_scan_scratch_bytes(uint64_t n) { return scan_layout(n).total; }

extern "C" int flip_inclusive_scan_u32(const uint32_t* in, uint32_t* out, uint64_t n, void* scratch, size_t bytes,
                                       void* stream) {
    if (n == 0) return FLIP_OK;
    if (!in || !out || n >= (1ull << 40)) {
        set_error_text("flip_inclusive_scan_u32: bad argument");
        return FLIP_ERR_ARG;
    }
    return launch_scan(0, in, out, n, scratch, bytes, as_stream(stream), nullptr, nullptr, nullptr, nullptr, kSpinLimit, 0);
}

// the binary architecture of the library's device code, as the runtime sees
// it for the scan kernel: 100 for sm_100a SASS
extern "C" int flip_binary_version(int* version) {
    if (!version) {
        set_error_text("flip_binary_version: null pointer");
        return FLIP_ERR_ARG;
    }
    cudaFuncAttributes a{};
    FLIP_CUDA_TRY(cudaFuncGetAttributes(&a, scan_kernel<0>));
    *version = a.binaryVersion;
    return FLIP_OK;
}

extern "C" size_t flip_segment_heads_scratch_bytes(uint64_t n) { return scan_layout(n).total; }

extern "C" int flip_segment_heads(const uint32_t* sorted_keys, uint64_t n, uint32_t* flags_scan, uint32_t* starts,
                                  uint32_t* node_keys, uint32_t* d_count, void* scratch, size_t bytes, void* stream) {
    if (!sorted_keys || !starts || !d_count || n >= (1ull << 32)) {
        set_error_text("flip_segment_heads: bad argument");
        return FLIP_ERR_ARG;
    }
    cudaStream_t s = as_stream(stream);
    if (n == 0) {
        FLIP_CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(uint32_t), s));
        return FLIP_OK;
    }
    return launch_scan(1, sorted_keys, flags_scan, n, scratch, bytes, s, starts, node_keys, d_count, nullptr, kSpinLimit,
                       0);
}

// The error word at the start of a sort or scan scratch (the same offset in
// both layouts) once the call's kernels on `stream` have finished.
extern "C" int flip_scratch_status(const void* scratch, void* stream, uint32_t* flags) {
    if (!scratch || !flags) {
        set_error_text("flip_scratch_status: null pointer");
        return FLIP_ERR_ARG;
    }
    cudaStream_t s = as_stream(stream);
    uint32_t w = 0;
    FLIP_CUDA_TRY(cudaMemcpyAsync(&w, scratch, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    FLIP_CUDA_TRY(cudaStreamSynchronize(s));
    *flags = w;
    if (w & DEVERR_LOOKBACK_TIMEOUT) {
        set_error_text("a decoupled look-back wait timed out; the sort or scan output is invalid");
        return FLIP_ERR_TIMEOUT;
    }
    return FLIP_OK;
}

// Runs the scan (which = 0) or the sort (which = 1) with tile 0 never
// claimed: the look-back of tile 1 then polls a status word that nothing
// publishes, gives up after spin_limit polls and sets the timeout bit, and
// every kernel still returns.  The status comes back through
// flip_scratch_status.  All accesses stay inside the caller's buffers and
// scratch (the unclaimed tile's outputs are simply not written).
extern "C" int flip_test_lookback_timeout(int which, const uint32_t* in, uint32_t* out_keys, uint32_t* out_vals,
                                          uint64_t n, uint32_t spin_limit, void* scratch, size_t scratch_bytes,
                                          void* stream, uint32_t* flags) {
    if (!in || !out_keys || !flags || (which == 1 && !out_vals) || (which != 0 && which != 1)) {
        set_error_text("flip_test_lookback_timeout: bad argument");
        return FLIP_ERR_ARG;
    }
    if (n <= (uint64_t)kScanTile || n >= (1ull << 30)) {
        set_error_text("flip_test_lookback_timeout: n must span at least two tiles of 4096 and stay below 2^30");
        return FLIP_ERR_ARG;
    }
    cudaStream_t s = as_stream(stream);
    int rc = which == 0 ? launch_scan(0, in, out_keys, n, scratch, scratch_bytes, s, nullptr, nullptr, nullptr, nullptr,
                                      spin_limit, 1)
                        : sort_pairs_ex(in, nullptr, out_keys, out_vals, n, 32, scratch, scratch_bytes, s, nullptr,
                                        spin_limit, 1);
    if (rc != FLIP_OK) return rc;
    return flip_scratch_status(scratch, stream, flags);
}

// ---------------------------------------------------------------------------
// Inclusive scan that allocates nothing.
//
// flip_inclusive_scan_u32 asks the caller for scratch, which most callers get
// from cudaMalloc.  Some callers cannot allocate: a host application that
// hands this library a fixed device-memory budget and owns every allocation
// (a DCC plug-in host, say), or a per-frame callback where cudaMalloc's
// implicit device synchronisation would stall the frame.  This variant keeps
// its look-back scratch in a file-scope device array instead, so the caller
// passes only the input and output buffers.
//
// The array holds the status words of at most kNoAllocScanMaxTiles tiles of
// 4096 elements, so n is limited to kNoAllocScanMaxN (2^28) elements; it is
// 512 KiB plus a 256-byte header on every GPU that loads the library, kept
// until the process exits.  Every call shares it and it keeps the previous
// call's contents, so each call first clears the words it will use; two
// calls whose kernels overlap on the GPU (different streams, or different
// host threads on one device) race on it and must be serialised by the
// caller.  The first call on a device looks up the array's device address
// (cudaGetSymbolAddress, with that device current); make that first call
// before any stream capture.  A failed lookup is not remembered: the next
// call tries again.
//
// A look-back wait that gives up sets bit 0 of the array's error word and the
// scan's output is then invalid.  The call cannot report that itself (it
// returns before the kernel runs); flip_inclusive_scan_u32_noalloc_status
// reads the word of the last call on the current device.
namespace flip {
constexpr uint64_t kNoAllocScanMaxN = 1ull << 28;
constexpr uint64_t kNoAllocScanMaxTiles = kNoAllocScanMaxN / kScanTile;  // 65536
constexpr int kNoAllocHeaderWords = 32;                                   // err + tile counter, 256 bytes
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned long long g_noalloc_scan_scratch[kNoAllocHeaderWords + kNoAllocScanMaxTiles];

static void* g_noalloc_scan_ptr[kNoAllocMaxDevices];
static std::mutex g_noalloc_scan_mutex;

__global__ void noalloc_scan_clear_kernel(unsigned long long* words, uint64_t count) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) words[i] = 0ull;
}

// the array's device address on the current device (looked up once per
// device; a failed lookup is retried by the next call)
static int noalloc_scan_words(const char* who, unsigned long long** words) {
    int dev = 0;
    FLIP_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) {
        set_error_text((std::string(who) + ": device ordinal beyond 63").c_str());
        return FLIP_ERR_DEVICE;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_scan_mutex);
    if (!g_noalloc_scan_ptr[dev]) {
        void* ptr = nullptr;
        cudaError_t ce = cudaGetSymbolAddress(&ptr, g_noalloc_scan_scratch);
        if (ce != cudaSuccess) return set_cuda_error(ce, "cudaGetSymbolAddress");
        g_noalloc_scan_ptr[dev] = ptr;
    }
    *words = (unsigned long long*)g_noalloc_scan_ptr[dev];
    return FLIP_OK;
}
}  // namespace flip

extern "C" int flip_inclusive_scan_u32_noalloc(const uint32_t* in, uint32_t* out, uint64_t n, void* stream) {
    using namespace flip;
    if (n == 0) return FLIP_OK;
    if (!in || !out) {
        set_error_text("flip_inclusive_scan_u32_noalloc: null buffer");
        return FLIP_ERR_ARG;
    }
    if (n > kNoAllocScanMaxN) {
        set_error_text("flip_inclusive_scan_u32_noalloc: n exceeds the maximum of 2^28 elements its static scratch covers;"
                       " use flip_inclusive_scan_u32 with caller scratch");
        return FLIP_ERR_ARG;
    }
    unsigned long long* words = nullptr;
    if (int rc = noalloc_scan_words("flip_inclusive_scan_u32_noalloc", &words)) return rc;
    const uint64_t tiles = (n + kScanTile - 1) / kScanTile;
    const uint64_t used = kNoAllocHeaderWords + tiles;
    cudaStream_t s = as_stream(stream);
    noalloc_scan_clear_kernel<<<(unsigned)((used + 255) / 256), 256, 0, s>>>(words, used);
    uint32_t* err = (uint32_t*)words;
    uint32_t* ctr = (uint32_t*)(words + 2);
    unsigned long long* status = words + kNoAllocHeaderWords;
    scan_kernel<0><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, out, n, status, ctr, err, nullptr, nullptr, nullptr,
                                                            kSpinLimit, 0);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

// The error word of the last flip_inclusive_scan_u32_noalloc on the current
// device: waits for `stream` (the stream of that call), then copies the word.
// Copying from the array needs no allocation either.
extern "C" int flip_inclusive_scan_u32_noalloc_status(void* stream, uint32_t* flags) {
    using namespace flip;
    if (!flags) {
        set_error_text("flip_inclusive_scan_u32_noalloc_status: null flags");
        return FLIP_ERR_ARG;
    }
    unsigned long long* words = nullptr;
    if (int rc = noalloc_scan_words("flip_inclusive_scan_u32_noalloc_status", &words)) return rc;
    cudaStream_t s = as_stream(stream);
    uint32_t w = 0;
    FLIP_CUDA_TRY(cudaMemcpyAsync(&w, words, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    FLIP_CUDA_TRY(cudaStreamSynchronize(s));
    *flags = w;
    if (w & DEVERR_LOOKBACK_TIMEOUT) {
        set_error_text("flip_inclusive_scan_u32_noalloc: a look-back wait timed out; the output is invalid");
        return FLIP_ERR_TIMEOUT;
    }
    return FLIP_OK;
}
