// sort.cu -- stable LSD radix sort of (u32 key, u32 value) pairs for sm_100a.
//
// Replaces the reference's 32-pass 1-bit split sort
// (engine/algorithms/radixSortKernels.cu:6-123), which moves ~80 bytes per
// key per pass and synchronises the host five times per pass.  Any stable
// sort yields the same (keys, permutation) pair, so the result is bit-exact.
//
// Structure (Adinets & Merrill's onesweep):
//   1. one upfront pass reads every key once and builds all digit histograms
//      (shared-memory atomics into one histogram per warp);
//   2. one kernel per 8-bit digit: each CTA claims the next tile of 6144 keys
//      from an atomic counter, ranks its keys per warp with match/ballot,
//      publishes its per-digit counts and resolves its global offsets with a
//      decoupled look-back over the predecessor tiles, then scatters through
//      shared memory so that global writes are runs of consecutive addresses.
// Traffic per key: 4 B (histogram) + per pass 8 B read + 8 B write.
#include "common.cuh"

namespace flip {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 24;
constexpr int kSortTile = kSortThreads * kSortItems;  // 6144 keys
constexpr int kRadix = 256;
constexpr int kMaxPasses = 4;
constexpr int kLook = 8;  // predecessors a look-back step reads at once

constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kValueMask = (1u << 30) - 1;

static inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

struct SortLayout {
    size_t err, hist, offsets, ctr, status, alt_k, alt_v, total;
};
static SortLayout sort_layout(uint64_t n) {
    SortLayout L;
    uint64_t tiles = (n + kSortTile - 1) / kSortTile;
    size_t o = 0;
    L.err = o; o = align_up(o + 16, 256);
    L.hist = o; o = align_up(o + sizeof(uint32_t) * kMaxPasses * kRadix, 256);
    L.offsets = o; o = align_up(o + sizeof(uint32_t) * kMaxPasses * kRadix, 256);
    L.ctr = o; o = align_up(o + sizeof(uint32_t) * kMaxPasses, 256);
    L.status = o; o = align_up(o + sizeof(uint32_t) * kMaxPasses * tiles * kRadix, 256);
    L.alt_k = o; o = align_up(o + sizeof(uint32_t) * n, 256);
    L.alt_v = o; o = align_up(o + sizeof(uint32_t) * n, 256);
    L.total = o;
    return L;
}

// ----------------------------------------------------------- histogram
// A block counts one contiguous chunk of the keys, kHistItems keys per
// thread and round (loads issued together, each warp reading 128 contiguous
// bytes), into its warps' own histograms: the digits of blob-concentrated
// keys would otherwise have every warp of the block adding into the same few
// words.  A key the whole warp shares (keys sorted or nearly so, as the
// tile keys of consecutive steps are) is counted for the warp, in registers
// while consecutive items keep it; otherwise each lane adds its own.  With
// nearly sorted keys a chunk holds few digits, so few of the block's bins
// reach the global histogram.
constexpr int kHistItems = 8;
constexpr uint64_t kHistRound = (uint64_t)kSortThreads * kHistItems;
__global__ void __launch_bounds__(kSortThreads, 6) sort_histogram_kernel(const uint32_t* __restrict__ keys, uint64_t n,
                                                                      int passes, uint64_t chunk,
                                                                      uint32_t* __restrict__ hist) {
    extern __shared__ uint32_t sh[];  // [kSortWarps][passes][kRadix]
    for (int i = threadIdx.x; i < kSortWarps * passes * kRadix; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const int warp = threadIdx.x >> 5;
    uint32_t* H = sh + warp * passes * kRadix;
    const uint64_t c0 = (uint64_t)blockIdx.x * chunk;
    const uint64_t c1 = c0 + chunk < n ? c0 + chunk : n;
    // a key the whole warp shares, over consecutive items, is counted in
    // registers (warp-uniform values) and reaches the histograms when the key
    // changes
    uint32_t run_key = 0u, run_cnt = 0u;
    const bool lane0 = (threadIdx.x & 31u) == 0u;
    // every thread of the block takes the same number of rounds (the votes
    // below need all lanes of a warp)
    for (uint64_t r0 = c0; r0 < c1; r0 += kHistRound) {
        const uint64_t i0 = r0 + threadIdx.x;
        uint32_t k[kHistItems];
#pragma unroll
        for (int j = 0; j < kHistItems; ++j) {
            const uint64_t i = i0 + (uint64_t)j * kSortThreads;
            k[j] = i < c1 ? keys[i] : 0u;
        }
#pragma unroll
        for (int j = 0; j < kHistItems; ++j) {
            const bool valid = i0 + (uint64_t)j * kSortThreads < c1;
            const uint32_t nvalid = (uint32_t)__popc(__ballot_sync(0xffffffffu, valid));
            const uint32_t k0 = __shfl_sync(0xffffffffu, k[j], 0);
            if (__all_sync(0xffffffffu, !valid || k[j] == k0)) {
                if (k0 != run_key || run_cnt == 0u) {
                    if (lane0 && run_cnt)
                        for (int p = 0; p < passes; ++p) atomicAdd(H + p * kRadix + ((run_key >> (8 * p)) & 0xFFu), run_cnt);
                    run_key = k0;
                    run_cnt = 0u;
                }
                run_cnt += nvalid;
            } else if (valid) {
                for (int p = 0; p < passes; ++p) atomicAdd(H + p * kRadix + ((k[j] >> (8 * p)) & 0xFFu), 1u);
            }
        }
    }
    if (lane0 && run_cnt)
        for (int p = 0; p < passes; ++p) atomicAdd(H + p * kRadix + ((run_key >> (8 * p)) & 0xFFu), run_cnt);
    __syncthreads();
    for (int i = threadIdx.x; i < passes * kRadix; i += blockDim.x) {
        uint32_t v = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) v += sh[w * passes * kRadix + i];
        if (v) atomicAdd(&hist[i], v);
    }
}

// exclusive scan of each pass's 256 bins -> global digit offsets
__global__ void sort_offsets_kernel(const uint32_t* __restrict__ hist, uint32_t* __restrict__ offsets) {
    __shared__ uint32_t sh[kRadix / 32 + 1];
    const int p = blockIdx.x;
    uint32_t v = hist[p * kRadix + threadIdx.x];
    uint32_t total;
    uint32_t ex = block_exclusive_scan<kRadix>(v, sh, &total);
    offsets[p * kRadix + threadIdx.x] = ex;
}

// ------------------------------------------------------------ onesweep
template <bool kIota>
__global__ void __launch_bounds__(kSortThreads, 3) onesweep_kernel(
    const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint32_t* __restrict__ kout,
    uint32_t* __restrict__ vout, uint64_t n, int shift, const uint32_t* __restrict__ offsets,
    uint32_t* __restrict__ status, uint32_t* __restrict__ tile_ctr, uint32_t* __restrict__ err, uint32_t spin_limit,
    uint32_t tile_base, uint32_t* __restrict__ head_dense, uint32_t head_limit) {
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_whist[kSortWarps][kRadix];  // warp counts, then warp offsets within the digit
    __shared__ uint32_t s_blk[kRadix];                // tile-local exclusive offset of each digit
    __shared__ uint32_t s_gbase[kRadix];              // global output base of each digit for this tile
    __shared__ uint32_t s_scan[kSortWarps + 1];
    extern __shared__ uint32_t s_stage[];  // the tile reordered: keys, then values
    uint32_t* s_keys = s_stage;
    uint32_t* s_vals = s_stage + kSortTile;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) s_tile = atomicAdd(tile_ctr, 1u) + tile_base;
    for (int i = tid; i < kSortWarps * kRadix; i += kSortThreads) (&s_whist[0][0])[i] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * kSortTile;

    uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        uint64_t idx = base + (uint64_t)warp * (kSortItems * 32) + i * 32 + lane;
        if (idx < n) {
            key[i] = kin[idx];
            val[i] = kIota ? (uint32_t)idx : vin[idx];
        } else {
            key[i] = 0xFFFFFFFFu;  // ranks after every valid key of digit 255 of this tile
            val[i] = 0u;
        }
    }
    // stable per-warp ranking, item order = input order
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        uint32_t d = (key[i] >> shift) & 0xFFu;
        uint32_t peers = __match_any_sync(0xffffffffu, d);
        uint32_t before = __popc(peers & lt);
        uint32_t prev = s_whist[warp][d];
        __syncwarp();
        if (before == 0) s_whist[warp][d] = prev + __popc(peers);
        __syncwarp();
        rank[i] = prev + before;
    }
    __syncthreads();

    // thread d owns digit d: warp offsets, tile count, look-back
    const int d = tid;
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
        uint32_t c = s_whist[w][d];
        s_whist[w][d] = run;
        run += c;
    }
    uint32_t* st = status + (size_t)tile * kRadix + d;
    uint32_t excl = 0;
    if (tile == 0) {
        st_relaxed_u32(st, kFlagPrefix | run);
    } else {
        st_relaxed_u32(st, kFlagAgg | run);
        // walk back kLook predecessors per poll (independent loads, one round
        // trip): add their aggregates in order up to the first inclusive
        // prefix; from a predecessor that has published nothing yet, poll
        // again (a bounded number of times)
        int64_t t = (int64_t)tile - 1;
        uint32_t spins = 0;
        while (t >= 0) {
            uint32_t sv[kLook];
#pragma unroll
            for (int j = 0; j < kLook; ++j)
                sv[j] = (t - j >= 0) ? ld_relaxed_u32(status + (size_t)(t - j) * kRadix + d) : 0u;
            int used = 0;
            bool prefix = false, wait = false;
#pragma unroll
            for (int j = 0; j < kLook; ++j) {
                if (prefix || wait || t - j < 0) continue;
                const uint32_t f = sv[j] & ~kValueMask;
                if (f == 0) {
                    wait = true;
                    continue;
                }
                excl += sv[j] & kValueMask;
                ++used;
                prefix = f == kFlagPrefix;
            }
            if (prefix) break;
            t -= used;
            if (wait && ++spins > spin_limit) {
                atomicOr(err, DEVERR_LOOKBACK_TIMEOUT);
                break;
            }
        }
        st_relaxed_u32(st, kFlagPrefix | ((excl + run) & kValueMask));
    }
    s_gbase[d] = offsets[d] + excl;
    uint32_t tot;
    s_blk[d] = block_exclusive_scan<kSortThreads>(run, s_scan, &tot);
    __syncthreads();

#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        uint32_t dd = (key[i] >> shift) & 0xFFu;
        uint32_t pos = s_blk[dd] + s_whist[warp][dd] + rank[i];
        s_keys[pos] = key[i];
        s_vals[pos] = val[i];
    }
    __syncthreads();
    const uint32_t valid = (uint32_t)((n - base) < (uint64_t)kSortTile ? (n - base) : kSortTile);
    for (uint32_t j = tid; j < valid; j += kSortThreads) {
        uint32_t k = s_keys[j];
        uint32_t dd = (k >> shift) & 0xFFu;
        uint32_t o = s_gbase[dd] + (j - s_blk[dd]);
        if (o < n) {  // always true unless a look-back wait timed out
            kout[o] = k;
            vout[o] = s_vals[j];
            // last pass: the tile's keys are sorted in full, so the first of a
            // run of equal keys here is a candidate head; the smallest
            // candidate over the tiles is the head
            if (head_dense && (j == 0 || s_keys[j - 1] != k) && k < head_limit) atomicMin(head_dense + k, o);
        }
    }
}

}  // namespace flip

using namespace flip;

extern "C" size_t flip_sort_pairs_scratch_bytes(uint64_t n) { return sort_layout(n).total; }

int flip::sort_pairs_ex(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out, uint32_t* vals_out,
                        uint64_t n, int key_bits, void* scratch, size_t scratch_bytes, cudaStream_t s,
                        uint32_t* err_accum, uint32_t spin_limit, uint32_t tile_base, uint32_t* head_dense,
                        uint32_t head_limit) {
    if (head_dense && head_limit) FLIP_CUDA_TRY(cudaMemsetAsync(head_dense, 0xFF, sizeof(uint32_t) * head_limit, s));
    if (n == 0) return FLIP_OK;
    if (!keys_in || !keys_out || !vals_out || !scratch || key_bits < 1 || key_bits > 32 || n >= (1ull << 30)) {
        set_error_text("flip_sort_pairs: bad argument (null pointer, key_bits outside 1..32 or n >= 2^30)");
        return FLIP_ERR_ARG;
    }
    SortLayout L = sort_layout(n);
    if (scratch_bytes < L.total) {
        set_error_text("flip_sort_pairs: scratch too small");
        return FLIP_ERR_ARG;
    }
    char* S = (char*)scratch;
    uint32_t* err = err_accum ? err_accum : (uint32_t*)(S + L.err);
    uint32_t* hist = (uint32_t*)(S + L.hist);
    uint32_t* offs = (uint32_t*)(S + L.offsets);
    uint32_t* ctr = (uint32_t*)(S + L.ctr);
    uint32_t* status = (uint32_t*)(S + L.status);
    uint32_t* ak = (uint32_t*)(S + L.alt_k);
    uint32_t* av = (uint32_t*)(S + L.alt_v);
    const int passes = (key_bits + 7) / 8;

    const uint64_t tiles = (n + kSortTile - 1) / kSortTile;
    if (tile_base >= tiles) {
        set_error_text("flip_sort_pairs: tile_base beyond the tile count");
        return FLIP_ERR_ARG;
    }
    const unsigned grid = (unsigned)(tiles - tile_base);
    // error word, histograms, offsets, counters and look-back words are
    // contiguous at the start of the scratch: clear them in one memset
    FLIP_CUDA_TRY(cudaMemsetAsync(S, 0, L.status + sizeof(uint32_t) * passes * tiles * kRadix, s));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    // the staging buffer may exceed the default 48 KB (once per device)
    static bool stage_attr[64] = {};
    if (dev >= 0 && dev < 64 && !stage_attr[dev]) {
        FLIP_CUDA_TRY(cudaFuncSetAttribute(onesweep_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           2 * kSortTile * (int)sizeof(uint32_t)));
        FLIP_CUDA_TRY(cudaFuncSetAttribute(onesweep_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           2 * kSortTile * (int)sizeof(uint32_t)));
        stage_attr[dev] = true;
    }
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // one wave: as many blocks as are resident at once
    const size_t hsmem = sizeof(uint32_t) * kSortWarps * passes * kRadix;
    int per_sm = 1;
    FLIP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sort_histogram_kernel, kSortThreads, hsmem));
    if (per_sm < 1) per_sm = 1;
    uint64_t hblocks = (n + kHistRound - 1) / kHistRound;
    if (hblocks > (uint64_t)sms * per_sm) hblocks = (uint64_t)sms * per_sm;
    const uint64_t hchunk = (n + hblocks * kHistRound - 1) / (hblocks * kHistRound) * kHistRound;
    hblocks = (n + hchunk - 1) / hchunk;
    sort_histogram_kernel<<<(unsigned)hblocks, kSortThreads, hsmem, s>>>(keys_in, n, passes, hchunk, hist);
    sort_offsets_kernel<<<passes, kRadix, 0, s>>>(hist, offs);
    // pass p writes `out` when (passes-1-p) is even, so the last pass lands in out
    const bool inplace_odd = (keys_in == keys_out || (vals_in && vals_in == vals_out)) && (passes % 2 == 1);
    const uint32_t* ck = keys_in;
    const uint32_t* cv = vals_in;
    for (int p = 0; p < passes; ++p) {
        bool to_out = ((passes - 1 - p) % 2 == 0) && !inplace_odd;
        if (inplace_odd) to_out = ((passes - 1 - p) % 2 == 1);
        uint32_t* ok = to_out ? keys_out : ak;
        uint32_t* ov = to_out ? vals_out : av;
        uint32_t* pstat = status + (size_t)p * tiles * kRadix;
        uint32_t* hd = p == passes - 1 ? head_dense : nullptr;
        constexpr int kStage = 2 * kSortTile * (int)sizeof(uint32_t);
        if (p == 0 && cv == nullptr)
            onesweep_kernel<true><<<grid, kSortThreads, kStage, s>>>(ck, nullptr, ok, ov, n, 8 * p, offs + p * kRadix, pstat,
                                                                ctr + p, err, spin_limit, tile_base, hd, head_limit);
        else
            onesweep_kernel<false><<<grid, kSortThreads, kStage, s>>>(ck, cv, ok, ov, n, 8 * p, offs + p * kRadix, pstat,
                                                                 ctr + p, err, spin_limit, tile_base, hd, head_limit);
        ck = ok;
        cv = ov;
    }
    if (inplace_odd) {  // odd pass count sorting in place: the result sits in the alternate buffers
        FLIP_CUDA_TRY(cudaMemcpyAsync(keys_out, ak, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
        FLIP_CUDA_TRY(cudaMemcpyAsync(vals_out, av, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
    }
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

extern "C" int flip_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                               uint32_t* vals_out, uint64_t n, int key_bits, void* scratch, size_t scratch_bytes,
                               void* stream) {
    return sort_pairs_ex(keys_in, vals_in, keys_out, vals_out, n, key_bits, scratch, scratch_bytes, as_stream(stream),
                         nullptr, kSpinLimit, 0);
}
