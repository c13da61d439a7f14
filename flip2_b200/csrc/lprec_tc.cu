// lprec_tc.cu -- tensor-core forward of the learned preconditioner's
// 16 -> 16 channel layers (dilated 3^3 convolutions, BF16 in, FP32
// accumulation in tensor memory, ReLU, BF16 out) as an implicit GEMM on the
// sm_100a UMMA unit (tcgen05.mma, kind::f16).
//
// One CTA works on one 8^3 tile of the active list at a time:
//   1. stage the tile's input box (8 + 2 dil)^3 voxels x 16 channels in
//      shared memory as two 8-channel planes, 16 B per voxel and plane, in
//      x-fastest order; voxels outside the box or in inactive tiles read 0;
//   2. one thread issues, for each z-slice of the tile and each of the 27
//      taps, one M=64 x N=16 x K=16 MMA: A = the 64 voxels (8 x, 8 y) of the
//      slice shifted by the tap, read straight from the box (rows 16 B apart,
//      8-row groups one box row apart, the two channel planes one plane
//      apart: the K-major no-swizzle canonical layout), B = the tap's 16 x 16
//      weights; the 27 products accumulate into one TMEM accumulator per
//      z-slice (8 slices x 16 columns);
//   3. the MMAs commit to an mbarrier; every warp waits on it (bounded), reads
//      its accumulators with tcgen05.ld, applies ReLU and stores BF16.
// An M=64 accumulator keeps row m in TMEM lane (m % 16) + 32 (m / 16) and
// column n at column n.  Waits are bounded: on a timeout the kernel sets an
// error flag, waits (bounded) for its MMAs, frees its TMEM and returns.
#include <cuda_bf16.h>
#include "common.cuh"
#include "lprec.cuh"

namespace flip {

namespace {
constexpr int kTcThreads = 256;   // 8 warps: 2 warpgroups for the TMEM reads
constexpr int kTcCols = 128;      // 8 z-slices x 16 FP32 columns
constexpr uint32_t kTcSpinLimit = 1u << 24;
constexpr uint32_t kInstrDesc = (1u << 4)           // D: FP32
                                | (1u << 7)         // A: BF16
                                | (1u << 10)        // B: BF16
                                | ((16u >> 3) << 17)  // N = 16
                                | ((64u >> 4) << 24);  // M = 64

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major, no swizzle: rows 16 B apart, 8-row groups sbo bytes apart, the two
// 16-byte K halves lbo bytes apart; descriptor version 1 (sm100)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

__device__ __forceinline__ void mma_f16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait; false on timeout
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (uint32_t it = 0; it < kTcSpinLimit; ++it)
        if (mbar_try_wait(mbar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tile_origin_tc(uint32_t key, const NatDims& D, int& ox, int& oy, int& oz) {
    ox = 8 * (int)(key % D.tx);
    oy = 8 * (int)((key / D.tx) % D.ty);
    oz = 8 * (int)(key / (D.tx * D.ty));
}
}  // namespace

// shared-memory footprint of one CTA for dilation DIL
template <int DIL>
struct TcSmem {
    static constexpr int B = 8 + 2 * DIL;                 // box edge
    static constexpr int kPlane = B * B * B * 16;         // bytes of one 8-channel plane
    static constexpr int kBox = 2 * kPlane;
    static constexpr int kW = 27 * 512;                   // 27 taps x (16 co x 16 ci) BF16
    static constexpr int kBytes = kBox + kW + 64;
};

template <int DIL>
__global__ void __launch_bounds__(kTcThreads) lp_mid_tc_kernel(LpGrid G, const __nv_bfloat16* __restrict__ wb,
                                                               const __nv_bfloat16* __restrict__ in,
                                                               __nv_bfloat16* __restrict__ out, int* __restrict__ err) {
    using S = TcSmem<DIL>;
    constexpr int B = S::B;
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* box = smem;
    unsigned char* wsm = smem + S::kBox;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + S::kBox + S::kW);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + S::kBox + S::kW + 16);
    __shared__ int s_abort;
    if (G.halt && *G.halt) return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // weights: global [tap][ci][co] -> per tap [ci/8][co][ci%8] (K-major B: rows = co)
    for (int e = tid; e < 27 * 256; e += kTcThreads) {
        const int tap = e >> 8, ci = (e >> 4) & 15, co = e & 15;
        const int off = tap * 512 + (ci >> 3) * 256 + co * 16 + (ci & 7) * 2;
        *reinterpret_cast<__nv_bfloat16*>(wsm + off) = wb[e];
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t box_s = smem_u32(box), w_s = smem_u32(wsm), mbar_s = smem_u32(mbar);
    const uint32_t n = *G.d_nact;
    uint32_t phase = 0;
    bool pending_mma = false;
    for (uint32_t t = blockIdx.x; t < n; t += gridDim.x) {
        const uint32_t key = G.act_tiles[t];
        int ox, oy, oz;
        tile_origin_tc(key, G.D, ox, oy, oz);
        // 1. input box, two 16-byte chunks per voxel
        for (int e = tid; e < 2 * B * B * B; e += kTcThreads) {
            const int c = e & 1, v = e >> 1;
            const int bx = v % B, by = (v / B) % B, bz = v / (B * B);
            const int gx = ox - DIL + bx, gy = oy - DIL + by, gz = oz - DIL + bz;
            uint4 val = make_uint4(0u, 0u, 0u, 0u);
            if (gx >= 0 && gy >= 0 && gz >= 0 && gx < G.D.nx && gy < G.D.ny && gz < G.D.nz) {
                const uint32_t tt = (uint32_t)((gx >> 3) + G.D.tx * ((gy >> 3) + G.D.ty * (gz >> 3)));
                if (G.tile_active[tt]) {
                    const uint32_t sl = (tt << 9) | (uint32_t)((gx & 7) | ((gy & 7) << 3) | ((gz & 7) << 6));
                    val = *reinterpret_cast<const uint4*>(in + (size_t)sl * 16 + c * 8);
                }
            }
            *reinterpret_cast<uint4*>(box + c * S::kPlane + v * 16) = val;
        }
        // make the generic-proxy writes visible to the tensor core's async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        // 2. 8 slices x 27 taps of M=64 N=16 K=16
        if (tid == 0) {
            for (int z = 0; z < 8; ++z) {
                for (int tap = 0; tap < 27; ++tap) {
                    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
                    const int bz = z + DIL + DIL * dz, by0 = DIL + DIL * dy, bx0 = DIL + DIL * dx;
                    const uint32_t aoff = (uint32_t)(((bz * B + by0) * B + bx0) * 16);
                    const uint64_t ad = umma_desc(box_s + aoff, S::kPlane, B * 16);
                    const uint64_t bd = umma_desc(w_s + tap * 512, 256, 128);
                    mma_f16(tmem + (uint32_t)(z * 16), ad, bd, kInstrDesc, tap > 0 ? 1u : 0u);
                }
            }
            mma_commit(mbar_s);
        }
        pending_mma = true;
        // 3. epilogue: warp w reads sub-partition w % 4 of slices w/4, w/4+2, w/4+4, w/4+6
        const bool ok = mbar_wait(mbar_s, phase);
        if (!ok) {
            if (lane == 0) atomicExch(&s_abort, 1);
        }
        __syncthreads();
        if (s_abort) break;
        pending_mma = false;
        phase ^= 1u;
        tc_fence_after();
        const int q = warp & 3;
        for (int zz = warp >> 2; zz < 8; zz += 2) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(zz * 16), v);
            if (lane < 16) {
                const int m = lane + 16 * q;  // row of the slice: x = m % 8, y = m / 8
                const uint32_t sl = (key << 9) | (uint32_t)((m & 7) | ((m >> 3) << 3) | (zz << 6));
                uint4 o0, o1;
                __nv_bfloat162* h0 = reinterpret_cast<__nv_bfloat162*>(&o0);
                __nv_bfloat162* h1 = reinterpret_cast<__nv_bfloat162*>(&o1);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    h0[k] = __floats2bfloat162_rn(fmaxf(v[2 * k], 0.0f), fmaxf(v[2 * k + 1], 0.0f));
                    h1[k] = __floats2bfloat162_rn(fmaxf(v[8 + 2 * k], 0.0f), fmaxf(v[8 + 2 * k + 1], 0.0f));
                }
                uint4* dst = reinterpret_cast<uint4*>(out + (size_t)sl * 16);
                dst[0] = o0;
                dst[1] = o1;
            }
        }
        tc_fence_before();
        __syncthreads();  // TMEM and the box are free for the next tile
        tc_fence_after();
    }
    if (s_abort) {
        if (tid == 0) atomicOr(err, 1);
        // bounded wait for the MMAs of the abandoned tile before freeing TMEM
        if (pending_mma) mbar_wait(mbar_s, phase);
        __syncthreads();
    }
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols) : "memory");
}

template <int DIL>
static int launch_mid_tc(const LpGrid& G, const __nv_bfloat16* wb, const __nv_bfloat16* in, __nv_bfloat16* out, int* err,
                         int sms, cudaStream_t st) {
    using S = TcSmem<DIL>;
    static bool attr_set = false;  // per process; the attribute is per function
    if (!attr_set) {
        FLIP_CUDA_TRY(cudaFuncSetAttribute(lp_mid_tc_kernel<DIL>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::kBytes));
        // all of the unified L1 as shared memory, so several CTAs fit per SM
        FLIP_CUDA_TRY(cudaFuncSetAttribute(lp_mid_tc_kernel<DIL>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        attr_set = true;
    }
    // CTAs per SM from the shared-memory budget (each CTA also holds 1 KB of
    // static and 1 KB of reserved shared memory); at most 4 x 128 TMEM columns
    int dev = 0, smem_sm = 0;
    FLIP_CUDA_TRY(cudaGetDevice(&dev));
    FLIP_CUDA_TRY(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    int per_sm = smem_sm / (S::kBytes + 2048);
    per_sm = per_sm < 1 ? 1 : (per_sm > 4 ? 4 : per_sm);
    lp_mid_tc_kernel<DIL><<<sms * per_sm, kTcThreads, S::kBytes, st>>>(G, wb, in, out, err);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

// ------------------------------------------------------------ small grids
// The 16 -> 16 layers on a small grid whose every tile is active (the
// coarsest level of the multilevel preconditioner, at most 4,096 voxels):
// one CTA per 128 consecutive voxels of the tile list.  The CTA gathers, for
// each of the 27 taps, its voxels' 16 input channels into an A operand of
// 128 rows (K-major, no swizzle: rows 16 B apart, 8-row groups 128 B apart,
// the two 8-channel halves 2 KB apart), so that one thread issues 27 MMAs of
// M=128 x N=16 x K=16 into one TMEM accumulator (row m in lane m).  Warps 0-3
// read their 32 lanes back, apply ReLU and store BF16.  Waits are bounded as
// in the per-tile kernel above.
namespace {
constexpr int kSmTcThreads = 256;
constexpr int kSmTcRows = 128;
constexpr int kSmTcA = 27 * kSmTcRows * 32;  // 27 taps x 128 rows x 16 BF16
constexpr int kSmTcW = 27 * 512;
constexpr int kSmTcBytes = kSmTcA + kSmTcW + 64;
constexpr uint32_t kInstrDescM128 = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);
}  // namespace

__global__ void __launch_bounds__(kSmTcThreads) lp_small_mid_tc_kernel(LpGrid G, const __nv_bfloat16* __restrict__ wb, int dil,
                                                                       const __nv_bfloat16* __restrict__ in,
                                                                       __nv_bfloat16* __restrict__ out, int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* asm_ = smem;
    unsigned char* wsm = smem + kSmTcA;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + kSmTcA + kSmTcW);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kSmTcA + kSmTcW + 16);
    __shared__ int s_abort;
    pdl_wait();
    if (G.halt && *G.halt) return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t nvox = *G.d_nact * 512u;
    const uint32_t v0 = blockIdx.x * kSmTcRows;
    if (v0 >= nvox) return;
    // weights: global [tap][ci][co] -> per tap [ci/8][co][ci%8]; 27 per thread,
    // loaded in batches of nine before they are stored
#pragma unroll
    for (int m0 = 0; m0 < 27; m0 += 9) {
        __nv_bfloat16 w[9];
#pragma unroll
        for (int j = 0; j < 9; ++j) w[j] = wb[tid + (m0 + j) * kSmTcThreads];
#pragma unroll
        for (int j = 0; j < 9; ++j) {
            const int e = tid + (m0 + j) * kSmTcThreads;
            const int tap = e >> 8, ci = (e >> 4) & 15, co = e & 15;
            *reinterpret_cast<__nv_bfloat16*>(wsm + tap * 512 + (ci >> 3) * 256 + co * 16 + (ci & 7) * 2) = w[j];
        }
    }
    // A: for each tap, row r = voxel v0 + r, half h = channels 8h .. 8h+7.
    // A thread keeps one (row, half) and walks the 27 taps: its voxel is
    // worked out once, and the taps' loads go out nine at a time.
    {
        const int h = tid & 1, r = tid >> 1;  // 256 threads = 128 rows x 2 halves
        const uint32_t vx = v0 + (uint32_t)r;
        int ci = 0, cj = 0, ck = 0;
        const bool have = vx < nvox;
        if (have) {
            int ox, oy, oz;
            tile_origin_tc(G.act_tiles[vx >> 9], G.D, ox, oy, oz);
            const int l = (int)(vx & 511u);
            ci = ox + (l & 7);
            cj = oy + ((l >> 3) & 7);
            ck = oz + (l >> 6);
        }
        unsigned char* dst = asm_ + h * (kSmTcRows * 16) + r * 16;
#pragma unroll
        for (int t0 = 0; t0 < 27; t0 += 9) {
            uint4 val[9];
#pragma unroll
            for (int j = 0; j < 9; ++j) {
                const int tap = t0 + j;
                const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
                const int gx = ci + dil * dx, gy = cj + dil * dy, gz = ck + dil * dz;
                val[j] = make_uint4(0u, 0u, 0u, 0u);
                if (have && gx >= 0 && gy >= 0 && gz >= 0 && gx < G.D.nx && gy < G.D.ny && gz < G.D.nz) {
                    const uint32_t tt = (uint32_t)((gx >> 3) + G.D.tx * ((gy >> 3) + G.D.ty * (gz >> 3)));
                    const uint32_t sl = (tt << 9) | (uint32_t)((gx & 7) | ((gy & 7) << 3) | ((gz & 7) << 6));
                    val[j] = *reinterpret_cast<const uint4*>(in + (size_t)sl * 16 + h * 8);
                }
            }
#pragma unroll
            for (int j = 0; j < 9; ++j) *reinterpret_cast<uint4*>(dst + (t0 + j) * (kSmTcRows * 32)) = val[j];
        }
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)), "r"(32)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // the generic-proxy stores above become visible to the tensor core's async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t a_s = smem_u32(asm_), w_s = smem_u32(wsm), mbar_s = smem_u32(mbar);
    if (tid == 0) {
        for (int tap = 0; tap < 27; ++tap) {
            const uint64_t ad = umma_desc(a_s + (uint32_t)(tap * kSmTcRows * 32), kSmTcRows * 16, 128);
            const uint64_t bd = umma_desc(w_s + (uint32_t)(tap * 512), 256, 128);
            mma_f16(tmem, ad, bd, kInstrDescM128, tap > 0 ? 1u : 0u);
        }
        mma_commit(mbar_s);
    }
    // one decision for the whole CTA: the TMEM reads below are warp-collective
    if (!mbar_wait(mbar_s, 0)) atomicExch(&s_abort, 1);
    __syncthreads();
    const bool ok = s_abort == 0;
    tc_fence_after();
    if (ok && warp < 4) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16), v);
        const uint32_t vx = v0 + (uint32_t)(32 * warp + lane);
        if (vx < nvox) {
            const uint32_t sl = (G.act_tiles[vx >> 9] << 9) | (vx & 511u);
            uint4 o0, o1;
            __nv_bfloat162* h0 = reinterpret_cast<__nv_bfloat162*>(&o0);
            __nv_bfloat162* h1 = reinterpret_cast<__nv_bfloat162*>(&o1);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                h0[k] = __floats2bfloat162_rn(fmaxf(v[2 * k], 0.0f), fmaxf(v[2 * k + 1], 0.0f));
                h1[k] = __floats2bfloat162_rn(fmaxf(v[8 + 2 * k], 0.0f), fmaxf(v[8 + 2 * k + 1], 0.0f));
            }
            uint4* dst = reinterpret_cast<uint4*>(out + (size_t)sl * 16);
            dst[0] = o0;
            dst[1] = o1;
        }
    }
    if (!ok) {
        if (tid == 0) atomicOr(err, 1);
        mbar_wait(mbar_s, 0);  // bounded: the MMAs before TMEM is freed
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32) : "memory");
}

// ------------------------------------------------------------ backward
// The backward pass of the 16 -> 16 layers on the tensor cores: a persistent
// grid whose CTAs take 128 consecutive voxels of the active list at a time.
//
// Input gradient (dgrad): Gin[v][ci] = relu'(Ain[v][ci]) sum_tap sum_co
// W[tap][ci][co] Gout[v - dil off(tap)][co], the forward GEMM with the taps
// mirrored and each tap's weights transposed.  The CTA gathers, for each tap,
// Gout at its voxels' mirrored neighbours (rounded to BF16; zero outside the
// grid or in an inactive tile) into a K-major A operand of 128 rows, as the
// small-grid forward does, and one thread issues 27 M=128 x N=16 x K=16 MMAs
// with B = the tap's W transposed.  Warps 0-3 read the FP32 sums back (row m
// in TMEM lane m), multiply by relu'(Ain) and store FP32.
//
// Weight gradient (wgrad), every layer: dW[tap][ci][co] = sum_v In[v + dil
// off(tap)][ci] Gout[v][co], a GEMM whose reduction runs over the voxels.
// The CTA gathers the layer's input at each tap's neighbours into
// A_buf[group][128 v][8 ci] (for a 16-channel input the groups are (tap,
// ci / 8)), which reads as an MN-major A: rows m = (group, ci % 8), groups of
// 8 rows 2 KB apart, the voxels along K 16 B apart.  Gout at its own voxels
// is staged as an MN-major B (voxels along K, co along N), as its BF16
// rounding and the BF16 rounding of the remainder, so that the products keep
// about 16 bits of Gout (and of the input layer's r/s, split the same way
// into two rows).  M=128 accumulators (16 row groups each) collect 8 K-steps
// of 16 voxels per chunk over all of the CTA's chunks; at the end warps 0-3
// add them into dW with FP32 atomics.  Waits are bounded as in the forward
// kernels.
namespace {
constexpr int kBwThreads = 256;
constexpr int kBwRows = 128;
constexpr int kDgA = 27 * kBwRows * 32;  // 27 taps x 128 rows x 16 BF16
constexpr int kDgBytes = kDgA + 27 * 512 + 64;
constexpr int kWgB = 2 * 2 * kBwRows * 16;  // B: high and low part x two co halves x 128 rows
constexpr uint32_t kInstrDescMN = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((16u >> 3) << 17) |
                                  ((128u >> 4) << 24);  // FP32 += BF16 x BF16, A and B MN-major, N=16, M=128

// slot of voxel vx of the active list and its cell (i, j, k)
__device__ __forceinline__ uint32_t bw_voxel(const LpGrid& G, uint32_t vx, int& i, int& j, int& k) {
    const uint32_t key = G.act_tiles[vx >> 9];
    int ox, oy, oz;
    tile_origin_tc(key, G.D, ox, oy, oz);
    const int l = (int)(vx & 511u);
    i = ox + (l & 7);
    j = oy + ((l >> 3) & 7);
    k = oz + (l >> 6);
    return (key << 9) | (uint32_t)l;
}
// slot of (i, j, k) if it is in the grid and in an active tile, else UINT32_MAX
__device__ __forceinline__ uint32_t bw_active(const LpGrid& G, int i, int j, int k) {
    if (i < 0 || j < 0 || k < 0 || i >= G.D.nx || j >= G.D.ny || k >= G.D.nz) return 0xFFFFFFFFu;
    const uint32_t t = (uint32_t)((i >> 3) + G.D.tx * ((j >> 3) + G.D.ty * (k >> 3)));
    if (!G.tile_active[t]) return 0xFFFFFFFFu;
    return (t << 9) | (uint32_t)((i & 7) | ((j & 7) << 3) | ((k & 7) << 6));
}
__device__ __forceinline__ uint4 bf16x8(const float4& a, const float4& b) {
    uint4 o;
    __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&o);
    h[0] = __floats2bfloat162_rn(a.x, a.y);
    h[1] = __floats2bfloat162_rn(a.z, a.w);
    h[2] = __floats2bfloat162_rn(b.x, b.y);
    h[3] = __floats2bfloat162_rn(b.z, b.w);
    return o;
}
// the BF16 rounding of what bf16x8 dropped
__device__ __forceinline__ uint4 bf16x8_rest(const float4& a, const float4& b, const uint4& hi) {
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&hi);
    const float2 h0 = __bfloat1622float2(h[0]), h1 = __bfloat1622float2(h[1]), h2 = __bfloat1622float2(h[2]),
                 h3 = __bfloat1622float2(h[3]);
    return bf16x8(make_float4(a.x - h0.x, a.y - h0.y, a.z - h1.x, a.w - h1.y),
                  make_float4(b.x - h2.x, b.y - h2.y, b.z - h3.x, b.w - h3.y));
}
__device__ __forceinline__ void tc_init(uint64_t* mbar, uint32_t* tslot, int* s_abort, uint32_t cols) {
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        *s_abort = 0;
    }
    if ((threadIdx.x >> 5) == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)), "r"(cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
}
}  // namespace

__global__ void __launch_bounds__(kBwThreads) lp_tc_dgrad_kernel(LpGrid G, const __nv_bfloat16* __restrict__ wb, int dil,
                                                                 const float* __restrict__ gout,
                                                                 const __nv_bfloat16* __restrict__ ain,
                                                                 float* __restrict__ gin, int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* abuf = smem;
    unsigned char* wsm = smem + kDgA;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + kDgA + 27 * 512);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kDgA + 27 * 512 + 16);
    __shared__ int s_abort;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t nvox = *G.d_nact * 512u;
    if (blockIdx.x * kBwRows >= nvox) return;
    // weights: global [tap][ci][co] -> per tap [co/8][ci][co%8] (K-major B: rows = ci, K = co)
    for (int e = tid; e < 27 * 256; e += kBwThreads) {
        const int tap = e >> 8, ci = (e >> 4) & 15, co = e & 15;
        *reinterpret_cast<__nv_bfloat16*>(wsm + tap * 512 + (co >> 3) * 256 + ci * 16 + (co & 7) * 2) = wb[e];
    }
    tc_init(mbar, tslot, &s_abort, 32);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t a_s = smem_u32(abuf), w_s = smem_u32(wsm), mbar_s = smem_u32(mbar);
    uint32_t phase = 0;
    bool pending = false;
    for (uint32_t v0 = blockIdx.x * kBwRows; v0 < nvox; v0 += gridDim.x * kBwRows) {
        {  // A: thread (row r, half h) gathers its voxel's 27 mirrored neighbours
            const int h = tid & 1, r = tid >> 1;
            const uint32_t vx = v0 + (uint32_t)r;
            int ci = 0, cj = 0, ck = 0;
            const bool have = vx < nvox;
            if (have) bw_voxel(G, vx, ci, cj, ck);
            unsigned char* dst = abuf + h * (kBwRows * 16) + r * 16;
#pragma unroll
            for (int t0 = 0; t0 < 27; t0 += 9) {
                float4 g0[9], g1[9];
#pragma unroll
                for (int jj = 0; jj < 9; ++jj) {
                    const int tap = t0 + jj;
                    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
                    g0[jj] = g1[jj] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    const uint32_t u = have ? bw_active(G, ci - dil * dx, cj - dil * dy, ck - dil * dz) : 0xFFFFFFFFu;
                    if (u != 0xFFFFFFFFu) {
                        const float4* p = reinterpret_cast<const float4*>(gout + (size_t)u * 16 + h * 8);
                        g0[jj] = p[0];
                        g1[jj] = p[1];
                    }
                }
#pragma unroll
                for (int jj = 0; jj < 9; ++jj)
                    *reinterpret_cast<uint4*>(dst + (t0 + jj) * (kBwRows * 32)) = bf16x8(g0[jj], g1[jj]);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
            for (int tap = 0; tap < 27; ++tap) {
                const uint64_t ad = umma_desc(a_s + (uint32_t)(tap * kBwRows * 32), kBwRows * 16, 128);
                const uint64_t bd = umma_desc(w_s + (uint32_t)(tap * 512), 256, 128);
                mma_f16(tmem, ad, bd, kInstrDescM128, tap > 0 ? 1u : 0u);
            }
            mma_commit(mbar_s);
        }
        pending = true;
        // one decision for the whole CTA: the TMEM reads below are warp-collective
        if (!mbar_wait(mbar_s, phase) && lane == 0) atomicExch(&s_abort, 1);
        __syncthreads();
        if (s_abort) break;
        pending = false;
        phase ^= 1u;
        tc_fence_after();
        if (warp < 4) {
            float acc[16];
            tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16), acc);
            const uint32_t vx = v0 + (uint32_t)(32 * warp + lane);
            if (vx < nvox) {
                const uint32_t sl = (G.act_tiles[vx >> 9] << 9) | (vx & 511u);
                const uint4* ap = reinterpret_cast<const uint4*>(ain + (size_t)sl * 16);
                const uint4 q0 = ap[0], q1 = ap[1];
                const __nv_bfloat16* a0 = reinterpret_cast<const __nv_bfloat16*>(&q0);
                const __nv_bfloat16* a1 = reinterpret_cast<const __nv_bfloat16*>(&q1);
                float o[16];
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    o[c] = __bfloat162float(a0[c]) > 0.0f ? acc[c] : 0.0f;
                    o[8 + c] = __bfloat162float(a1[c]) > 0.0f ? acc[8 + c] : 0.0f;
                }
                float4* dp = reinterpret_cast<float4*>(gin + (size_t)sl * 16);
#pragma unroll
                for (int m = 0; m < 4; ++m) dp[m] = make_float4(o[4 * m], o[4 * m + 1], o[4 * m + 2], o[4 * m + 3]);
            }
        }
        tc_fence_before();
        __syncthreads();  // TMEM and the A operand are free for the next chunk
        tc_fence_after();
    }
    if (s_abort) {
        if (tid == 0) atomicOr(err, 1);
        if (pending) mbar_wait(mbar_s, phase);  // bounded: the MMAs before TMEM is freed
        __syncthreads();
    }
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32) : "memory");
}

// Weight-gradient layouts per layer (WG): the A row groups of 8 (MN-major,
// 2 KB apart), the accumulators, and the B parts.
//   WG 1 (16 -> 16): groups (tap, half) = 54, rows ci % 8; B = Gout [slot][16]
//                    as a high and a low part (two MMAs per step).
//   WG 2 (16 -> 1):  groups as WG 1; B = s gz [slot] with its high part in
//                    column 0 and its low part in column 1 (one MMA per step);
//                    dW = column 0 + column 1.  Voxels: the output list.
//   WG 0 (3 -> 16):  groups tap = 27, rows [r/s high, fluid, solid, r/s low,
//                    0, 0, 0, 0] from the input channels; B as WG 1;
//                    dW[.][0] = row 0 + row 3.
template <int WG>
struct WgShape {
    static constexpr int kGroups = WG == 0 ? 32 : 64;  // padded to whole M=128 accumulators
    static constexpr int kUsed = WG == 0 ? 27 : 54;
    static constexpr int kAcc = kGroups / 16;
    static constexpr int kParts = WG == 2 ? 1 : 2;
    static constexpr int kA = kGroups * kBwRows * 16;
    static constexpr int kBytes = kA + kWgB + 64;
};

template <int WG>
__global__ void __launch_bounds__(kBwThreads) lp_tc_wgrad_kernel(LpGrid G, int dil, const float* __restrict__ gout,
                                                                 const __nv_bfloat16* __restrict__ ain,
                                                                 const float* __restrict__ d_inv_s, float sign,
                                                                 const uint32_t* __restrict__ tiles,
                                                                 const uint32_t* __restrict__ d_n, float* __restrict__ dw,
                                                                 int* __restrict__ err) {
    using S = WgShape<WG>;
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* abuf = smem;
    unsigned char* bbuf = smem + S::kA;  // [part][co half][128 v][8 co]
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + S::kA + kWgB);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + S::kA + kWgB + 16);
    __shared__ int s_abort;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t nvox = *d_n * 512u;
    if (blockIdx.x * kBwRows >= nvox) return;
    const float inv_s = (WG == 1) ? 1.0f : *d_inv_s;
    // the row groups past the used ones stay zero, and so do the B columns
    // that WG 2 leaves empty
    for (int e = tid; e < (S::kGroups - S::kUsed) * kBwRows; e += kBwThreads)
        *reinterpret_cast<uint4*>(abuf + S::kUsed * kBwRows * 16 + e * 16) = make_uint4(0u, 0u, 0u, 0u);
    if (WG == 2)
        for (int e = tid; e < kWgB / 16; e += kBwThreads) *reinterpret_cast<uint4*>(bbuf + e * 16) = make_uint4(0u, 0u, 0u, 0u);
    tc_init(mbar, tslot, &s_abort, 64);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t a_s = smem_u32(abuf), b_s = smem_u32(bbuf), mbar_s = smem_u32(mbar);
    uint32_t phase = 0;
    bool pending = false, any = false;
    for (uint32_t v0 = blockIdx.x * kBwRows; v0 < nvox; v0 += gridDim.x * kBwRows) {
        {
            const int h = tid & 1, r = tid >> 1;
            const uint32_t vx = v0 + (uint32_t)r;
            int ci = 0, cj = 0, ck = 0;
            const bool have = vx < nvox;
            uint32_t self = 0;
            if (have) {
                const uint32_t key = tiles[vx >> 9];
                int ox, oy, oz;
                tile_origin_tc(key, G.D, ox, oy, oz);
                const int l = (int)(vx & 511u);
                ci = ox + (l & 7);
                cj = oy + ((l >> 3) & 7);
                ck = oz + (l >> 6);
                self = (key << 9) | (uint32_t)l;
            }
            // B: the output gradient at the voxel itself
            if (WG == 2) {
                if (h == 0) {
                    const float g = have ? gout[self] * (sign / inv_s) : 0.0f;
                    const __nv_bfloat16 hi = __float2bfloat16_rn(g);
                    const __nv_bfloat16 lo = __float2bfloat16_rn(g - __bfloat162float(hi));
                    __nv_bfloat16* row = reinterpret_cast<__nv_bfloat16*>(bbuf + r * 16);
                    row[0] = hi;
                    row[1] = lo;
                }
            } else {
                float4 g0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), g1 = g0;
                if (have) {
                    const float4* p = reinterpret_cast<const float4*>(gout + (size_t)self * 16 + h * 8);
                    g0 = p[0];
                    g1 = p[1];
                }
                const uint4 hi = bf16x8(g0, g1);
                *reinterpret_cast<uint4*>(bbuf + h * (kBwRows * 16) + r * 16) = hi;
                *reinterpret_cast<uint4*>(bbuf + 2 * kBwRows * 16 + h * (kBwRows * 16) + r * 16) = bf16x8_rest(g0, g1, hi);
            }
            if (WG == 0) {
                // A: the three input channels at taps 14 h .. 14 h + 13, group = tap
                for (int tap = 14 * h; tap < 14 * h + 14 && tap < 27; ++tap) {
                    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
                    const uint32_t u = have ? bw_active(G, ci + dil * dx, cj + dil * dy, ck + dil * dz) : 0xFFFFFFFFu;
                    float x = 0.0f, fl = 0.0f, so = 0.0f;
                    if (u != 0xFFFFFFFFu) {
                        const uint8_t t = G.type[u];
                        fl = t == kFluid ? 1.0f : 0.0f;
                        so = t == kSolid ? 1.0f : 0.0f;
                        x = (t == kFluid && G.r) ? G.r[u] * inv_s : 0.0f;
                    }
                    const __nv_bfloat16 xh = __float2bfloat16_rn(x);
                    const float xl = x - __bfloat162float(xh);
                    uint4 v;
                    __nv_bfloat162* hv = reinterpret_cast<__nv_bfloat162*>(&v);
                    hv[0] = __halves2bfloat162(xh, __float2bfloat16_rn(fl));
                    hv[1] = __floats2bfloat162_rn(so, xl);
                    hv[2] = hv[3] = __floats2bfloat162_rn(0.0f, 0.0f);
                    *reinterpret_cast<uint4*>(abuf + tap * (kBwRows * 16) + r * 16) = v;
                }
            } else {
                // A: the activations at the voxel's 27 neighbours, group (tap, h)
                unsigned char* dst = abuf + h * (kBwRows * 16) + r * 16;
#pragma unroll
                for (int t0 = 0; t0 < 27; t0 += 9) {
                    uint4 val[9];
#pragma unroll
                    for (int jj = 0; jj < 9; ++jj) {
                        const int tap = t0 + jj;
                        const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
                        val[jj] = make_uint4(0u, 0u, 0u, 0u);
                        const uint32_t u = have ? bw_active(G, ci + dil * dx, cj + dil * dy, ck + dil * dz) : 0xFFFFFFFFu;
                        if (u != 0xFFFFFFFFu) val[jj] = *reinterpret_cast<const uint4*>(ain + (size_t)u * 16 + h * 8);
                    }
#pragma unroll
                    for (int jj = 0; jj < 9; ++jj) *reinterpret_cast<uint4*>(dst + (t0 + jj) * (kBwRows * 32)) = val[jj];
                }
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
            for (int jm = 0; jm < S::kAcc; ++jm) {
                for (int ks = 0; ks < kBwRows / 16; ++ks) {
                    // A: row groups 16 jm .. 16 jm + 15 (2 KB apart), voxels 16 ks .. 16 ks + 15
                    const uint64_t ad = umma_desc(a_s + (uint32_t)(jm * 16 * kBwRows * 16 + ks * 256), 128, kBwRows * 16);
                    for (int part = 0; part < S::kParts; ++part) {
                        const uint64_t bd = umma_desc(b_s + (uint32_t)(part * 2 * kBwRows * 16 + ks * 256), 128, kBwRows * 16);
                        mma_f16(tmem + (uint32_t)(16 * jm), ad, bd, kInstrDescMN, (any || ks > 0 || part > 0) ? 1u : 0u);
                    }
                }
            }
            mma_commit(mbar_s);
        }
        any = true;
        pending = true;
        if (!mbar_wait(mbar_s, phase) && lane == 0) atomicExch(&s_abort, 1);
        __syncthreads();
        if (s_abort) break;
        pending = false;
        phase ^= 1u;
        tc_fence_before();
        __syncthreads();  // the MMAs are done with A and B: the next chunk may overwrite them
        tc_fence_after();
    }
    if (!s_abort && any && warp < 4) {
        tc_fence_after();
        for (int jm = 0; jm < S::kAcc; ++jm) {
            float acc[16];
            tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(16 * jm), acc);
            const int m = 32 * warp + lane;
            const int g = 16 * jm + m / 8;  // this lane's row group
            if (g >= S::kUsed) continue;
            if (WG == 0) {
                // rows r/s high (0) and low (3) both feed channel 0
                const int c = m & 7;
                const int cin = c == 3 ? 0 : c;
                if (c > 3) continue;
                float* d = dw + (g * 3 + cin) * 16;
#pragma unroll
                for (int co = 0; co < 16; ++co)
                    if (acc[co] != 0.0f) atomicAdd(d + co, acc[co]);
            } else {
                const int tap = g >> 1, cin = 8 * (g & 1) + (m & 7);
                if (WG == 2) {
                    const float v = acc[0] + acc[1];
                    if (v != 0.0f) atomicAdd(dw + tap * 16 + cin, v);
                } else {
                    float* d = dw + (tap * 16 + cin) * 16;
#pragma unroll
                    for (int co = 0; co < 16; ++co)
                        if (acc[co] != 0.0f) atomicAdd(d + co, acc[co]);
                }
            }
        }
    }
    if (s_abort) {
        if (tid == 0) atomicOr(err, 1);
        if (pending) mbar_wait(mbar_s, phase);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64) : "memory");
}

int lp_mid_dgrad_tc(const LpGrid& G, const __nv_bfloat16* wb, int dil, const float* gout, const __nv_bfloat16* ain,
                    float* gin, int* err, int sms, cudaStream_t st) {
    static bool attr_set = false;  // per process; the attribute is per function
    if (!attr_set) {
        FLIP_CUDA_TRY(cudaFuncSetAttribute(lp_tc_dgrad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kDgBytes));
        attr_set = true;
    }
    lp_tc_dgrad_kernel<<<sms, kBwThreads, kDgBytes, st>>>(G, wb, dil, gout, ain, gin, err);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

template <int WG>
static int launch_wgrad_tc(const LpGrid& G, int dil, const float* gout, const __nv_bfloat16* ain, const float* d_inv_s,
                           float sign, const uint32_t* tiles, const uint32_t* d_n, float* dw, int* err, int sms,
                           cudaStream_t st) {
    static bool attr_set = false;  // per process; the attribute is per function
    if (!attr_set) {
        FLIP_CUDA_TRY(cudaFuncSetAttribute(lp_tc_wgrad_kernel<WG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           WgShape<WG>::kBytes));
        attr_set = true;
    }
    lp_tc_wgrad_kernel<WG><<<sms, kBwThreads, WgShape<WG>::kBytes, st>>>(G, dil, gout, ain, d_inv_s, sign, tiles, d_n, dw,
                                                                          err);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int lp_in_wgrad_tc(const LpGrid& G, int dil, const float* gout, const float* d_inv_s, float* dw, int* err, int sms,
                   cudaStream_t st) {
    return launch_wgrad_tc<0>(G, dil, gout, nullptr, d_inv_s, 1.0f, G.act_tiles, G.d_nact, dw, err, sms, st);
}
int lp_mid_wgrad_tc(const LpGrid& G, int dil, const float* gout, const __nv_bfloat16* ain, float* dw, int* err, int sms,
                    cudaStream_t st) {
    return launch_wgrad_tc<1>(G, dil, gout, ain, nullptr, 1.0f, G.act_tiles, G.d_nact, dw, err, sms, st);
}
int lp_out_wgrad_tc(const LpGrid& G, int dil, const float* gz, const __nv_bfloat16* ain, const float* d_inv_s, float sign,
                    float* dw, int* err, int sms, cudaStream_t st) {
    return launch_wgrad_tc<2>(G, dil, gz, ain, d_inv_s, sign, G.out_tiles, G.d_nout, dw, err, sms, st);
}

int lp_small_mid_forward_tc(const LpGrid& G, const __nv_bfloat16* wb, int dil, const __nv_bfloat16* in, __nv_bfloat16* out,
                            int* err, uint32_t ntiles, cudaStream_t st) {
    static bool attr_set = false;  // per process; the attribute is per function
    if (!attr_set) {
        FLIP_CUDA_TRY(cudaFuncSetAttribute(lp_small_mid_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmTcBytes));
        attr_set = true;
    }
    const int grid = (int)((ntiles * 512u + kSmTcRows - 1) / kSmTcRows);
    FLIP_CUDA_TRY(pdl_launch(lp_small_mid_tc_kernel, grid, kSmTcThreads, kSmTcBytes, st, G, wb, dil, in, out, err));
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int lp_mid_forward_tc(const LpGrid& G, const __nv_bfloat16* wb, int dil, const __nv_bfloat16* in, __nv_bfloat16* out,
                      int* err, int sms, cudaStream_t st) {
    switch (dil) {
    case 1: return launch_mid_tc<1>(G, wb, in, out, err, sms, st);
    case 2: return launch_mid_tc<2>(G, wb, in, out, err, sms, st);
    case 4: return launch_mid_tc<4>(G, wb, in, out, err, sms, st);
    default: return FLIP_ERR_ARG;
    }
}

}  // namespace flip
