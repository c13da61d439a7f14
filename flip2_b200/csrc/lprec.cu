// lprec.cu -- forward and backward kernels of the learned preconditioner on
// CUDA cores (FP32 accumulation of BF16 weights and activations).
//
// Every kernel walks a tile list with one CTA of 512 threads per 8^3 tile
// and one thread per voxel.  A neighbour u = v + dil*offset contributes only
// if it lies in the box and in an active tile (its activations were written
// this solve); elsewhere it reads as zero (zero padding).
#include "common.cuh"
#include "lprec.cuh"

namespace flip {

__device__ __forceinline__ void tap_off(int tap, int& dx, int& dy, int& dz) {
    dz = tap / 9 - 1;
    dy = (tap / 3) % 3 - 1;
    dx = tap % 3 - 1;
}
__device__ __forceinline__ uint32_t lslot(int i, int j, int k, const NatDims& D) {
    uint32_t t = (uint32_t)((i >> 3) + D.tx * ((j >> 3) + D.ty * (k >> 3)));
    return (t << 9) | (uint32_t)((i & 7) | ((j & 7) << 3) | ((k & 7) << 6));
}
// slot of (i,j,k) if it is in the box and in an active tile, else UINT32_MAX
__device__ __forceinline__ uint32_t active_slot(int i, int j, int k, const LpGrid& G) {
    const NatDims& D = G.D;
    if (i < 0 || j < 0 || k < 0 || i >= D.nx || j >= D.ny || k >= D.nz) return 0xFFFFFFFFu;
    uint32_t t = (uint32_t)((i >> 3) + D.tx * ((j >> 3) + D.ty * (k >> 3)));
    if (!G.tile_active[t]) return 0xFFFFFFFFu;
    return (t << 9) | (uint32_t)((i & 7) | ((j & 7) << 3) | ((k & 7) << 6));
}
__device__ __forceinline__ void tile_origin(uint32_t key, const NatDims& D, int& ox, int& oy, int& oz) {
    ox = 8 * (int)(key % D.tx);
    oy = 8 * (int)((key / D.tx) % D.ty);
    oz = 8 * (int)(key / (D.tx * D.ty));
}
// the three input channels at slot u: r/s on fluid cells, fluid flag, solid flag
__device__ __forceinline__ void input_channels(const LpGrid& G, uint32_t u, float inv_s, float (&in)[3]) {
    const uint8_t t = G.type[u];
    const bool fl = t == kFluid;
    in[0] = (fl && G.r) ? G.r[u] * inv_s : 0.0f;
    in[1] = fl ? 1.0f : 0.0f;
    in[2] = (t == kSolid) ? 1.0f : 0.0f;
}
__device__ __forceinline__ void load16(const __nv_bfloat16* a, uint32_t u, float (&x)[16]) {
    const uint4* p = reinterpret_cast<const uint4*>(a + (size_t)u * 16);
    uint4 q0 = p[0], q1 = p[1];
    const __nv_bfloat162* h0 = reinterpret_cast<const __nv_bfloat162*>(&q0);
    const __nv_bfloat162* h1 = reinterpret_cast<const __nv_bfloat162*>(&q1);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        float2 f0 = __bfloat1622float2(h0[m]), f1 = __bfloat1622float2(h1[m]);
        x[2 * m] = f0.x; x[2 * m + 1] = f0.y;
        x[8 + 2 * m] = f1.x; x[8 + 2 * m + 1] = f1.y;
    }
}
__device__ __forceinline__ void store16(__nv_bfloat16* a, uint32_t u, const float (&x)[16]) {
    uint4 q0, q1;
    __nv_bfloat162* h0 = reinterpret_cast<__nv_bfloat162*>(&q0);
    __nv_bfloat162* h1 = reinterpret_cast<__nv_bfloat162*>(&q1);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        h0[m] = __floats2bfloat162_rn(x[2 * m], x[2 * m + 1]);
        h1[m] = __floats2bfloat162_rn(x[8 + 2 * m], x[8 + 2 * m + 1]);
    }
    uint4* p = reinterpret_cast<uint4*>(a + (size_t)u * 16);
    p[0] = q0;
    p[1] = q1;
}

// ---------------------------------------------------------------- forward
// layer 0: 3 -> 16, ReLU
__global__ void __launch_bounds__(512) lp_in_kernel(LpGrid G, const __nv_bfloat16* __restrict__ wb, int dil,
                                                    const float* __restrict__ d_inv_s, __nv_bfloat16* __restrict__ out) {
    if (G.halt && *G.halt) return;
    __shared__ float W[27 * 3 * 16];
    for (int i = threadIdx.x; i < 27 * 3 * 16; i += 512) W[i] = __bfloat162float(wb[i]);
    __syncthreads();
    const float inv_s = *d_inv_s;
    const uint32_t n = *G.d_nact;
    const int li = threadIdx.x & 7, lj = (threadIdx.x >> 3) & 7, lk = threadIdx.x >> 6;
    for (uint32_t t = blockIdx.x; t < n; t += gridDim.x) {
        const uint32_t key = G.act_tiles[t];
        int ox, oy, oz;
        tile_origin(key, G.D, ox, oy, oz);
        const int i = ox + li, j = oy + lj, k = oz + lk;
        float acc[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) acc[c] = 0.0f;
        for (int tap = 0; tap < 27; ++tap) {
            int dx, dy, dz;
            tap_off(tap, dx, dy, dz);
            const uint32_t u = active_slot(i + dil * dx, j + dil * dy, k + dil * dz, G);
            if (u == 0xFFFFFFFFu) continue;
            float in[3];
            input_channels(G, u, inv_s, in);
#pragma unroll
            for (int ci = 0; ci < 3; ++ci)
#pragma unroll
                for (int co = 0; co < 16; ++co) acc[co] = fmaf(W[(tap * 3 + ci) * 16 + co], in[ci], acc[co]);
        }
#pragma unroll
        for (int c = 0; c < 16; ++c) acc[c] = fmaxf(acc[c], 0.0f);
        store16(out, (key << 9) | threadIdx.x, acc);
    }
}

// layers 1, 2: 16 -> 16, ReLU
__global__ void __launch_bounds__(512) lp_mid_kernel(LpGrid G, const __nv_bfloat16* __restrict__ wb, int dil,
                                                     const __nv_bfloat16* __restrict__ in, __nv_bfloat16* __restrict__ out) {
    if (G.halt && *G.halt) return;
    __shared__ float W[27 * 16 * 16];
    for (int i = threadIdx.x; i < 27 * 256; i += 512) W[i] = __bfloat162float(wb[i]);
    __syncthreads();
    const uint32_t n = *G.d_nact;
    const int li = threadIdx.x & 7, lj = (threadIdx.x >> 3) & 7, lk = threadIdx.x >> 6;
    for (uint32_t t = blockIdx.x; t < n; t += gridDim.x) {
        const uint32_t key = G.act_tiles[t];
        int ox, oy, oz;
        tile_origin(key, G.D, ox, oy, oz);
        const int i = ox + li, j = oy + lj, k = oz + lk;
        float acc[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) acc[c] = 0.0f;
        for (int tap = 0; tap < 27; ++tap) {
            int dx, dy, dz;
            tap_off(tap, dx, dy, dz);
            const uint32_t u = active_slot(i + dil * dx, j + dil * dy, k + dil * dz, G);
            if (u == 0xFFFFFFFFu) continue;
            float x[16];
            load16(in, u, x);
            const float* w = W + tap * 256;
#pragma unroll
            for (int ci = 0; ci < 16; ++ci)
#pragma unroll
                for (int co = 0; co < 16; ++co) acc[co] = fmaf(w[ci * 16 + co], x[ci], acc[co]);
        }
#pragma unroll
        for (int c = 0; c < 16; ++c) acc[c] = fmaxf(acc[c], 0.0f);
        store16(out, (key << 9) | threadIdx.x, acc);
    }
}

// layer 3: 16 -> 1 on fluid cells.  raw: z = f (the zero-residual pass);
// else z = s (f - f0[v]) with f0 optional
__global__ void __launch_bounds__(512) lp_out_kernel(LpGrid G, const __nv_bfloat16* __restrict__ wb, int dil,
                                                     const __nv_bfloat16* __restrict__ in, const float* __restrict__ d_inv_s,
                                                     const float* __restrict__ f0, int raw, float* __restrict__ z) {
    if (G.halt && *G.halt) return;
    __shared__ float W[27 * 16];
    for (int i = threadIdx.x; i < 27 * 16; i += 512) W[i] = __bfloat162float(wb[i]);
    __syncthreads();
    const float s = 1.0f / *d_inv_s;
    const uint32_t n = *G.d_nout;
    const int li = threadIdx.x & 7, lj = (threadIdx.x >> 3) & 7, lk = threadIdx.x >> 6;
    for (uint32_t t = blockIdx.x; t < n; t += gridDim.x) {
        const uint32_t key = G.out_tiles[t];
        const uint32_t v = (key << 9) | threadIdx.x;
        float acc = 0.0f;
        if (G.type[v] == kFluid) {
            int ox, oy, oz;
            tile_origin(key, G.D, ox, oy, oz);
            const int i = ox + li, j = oy + lj, k = oz + lk;
            for (int tap = 0; tap < 27; ++tap) {
                int dx, dy, dz;
                tap_off(tap, dx, dy, dz);
                const uint32_t u = active_slot(i + dil * dx, j + dil * dy, k + dil * dz, G);
                if (u == 0xFFFFFFFFu) continue;
                float x[16];
                load16(in, u, x);
#pragma unroll
                for (int ci = 0; ci < 16; ++ci) acc = fmaf(W[tap * 16 + ci], x[ci], acc);
            }
            if (!raw) acc = (acc - (f0 ? f0[v] : 0.0f)) * s;
        }
        z[v] = acc;
    }
}

// ------------------------------------------------- forward on small grids
// The coarsest level of the multilevel preconditioner has at most eight
// tiles (4,096 voxels).  One CTA per tile would occupy eight SMs and chain 27
// dependent tap loads per thread, so these kernels give a CTA 16 voxels:
// first the CTA gathers the inputs of all 27 taps of its voxels into shared
// memory in one round of independent loads, then 16 threads per voxel (one
// per output channel, or one per input channel for the last layer) compute
// from shared memory.  Every tile of the small grid is active, so a tap
// only tests the grid bounds.
constexpr int kSmallThreads = 256;
constexpr int kSmallVox = 16;

__device__ __forceinline__ uint32_t small_slot(int i, int j, int k, const NatDims& D) {
    if (i < 0 || j < 0 || k < 0 || i >= D.nx || j >= D.ny || k >= D.nz) return 0xFFFFFFFFu;
    return lslot(i, j, k, D);
}
// cell (i, j, k) and slot of the CTA's voxel q (0..15), false past the grid
__device__ __forceinline__ bool small_voxel(const LpGrid& G, int q, uint32_t& v, int& i, int& j, int& k) {
    const uint32_t vx = blockIdx.x * kSmallVox + q;
    if (vx >= *G.d_nact * 512u) return false;
    const uint32_t key = G.act_tiles[vx >> 9];
    int ox, oy, oz;
    tile_origin(key, G.D, ox, oy, oz);
    const int l = (int)(vx & 511u);
    i = ox + (l & 7);
    j = oy + ((l >> 3) & 7);
    k = oz + (l >> 6);
    v = (key << 9) | (uint32_t)l;
    return true;
}
// X[q][tap][16] <- the 16 BF16 channels of in at tap of voxel q (0 outside)
__device__ __forceinline__ void small_gather16(const LpGrid& G, int dil, const __nv_bfloat16* __restrict__ in, uint4* X) {
    for (int e = threadIdx.x; e < kSmallVox * 27 * 2; e += kSmallThreads) {
        const int q = e / 54, tap = (e % 54) >> 1, half = e & 1;
        uint32_t v;
        int i, j, k, dx, dy, dz;
        uint4 val = make_uint4(0u, 0u, 0u, 0u);
        if (small_voxel(G, q, v, i, j, k)) {
            tap_off(tap, dx, dy, dz);
            const uint32_t u = small_slot(i + dil * dx, j + dil * dy, k + dil * dz, G.D);
            if (u != 0xFFFFFFFFu) val = reinterpret_cast<const uint4*>(in + (size_t)u * 16)[half];
        }
        X[e] = val;
    }
}
__device__ __forceinline__ void unpack8(const uint4& q, float* x) {
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&q);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const float2 f = __bfloat1622float2(h[m]);
        x[2 * m] = f.x;
        x[2 * m + 1] = f.y;
    }
}

// layer 0 (3 -> 16, ReLU); r = nullptr in G gives the zero-residual pass
__global__ void __launch_bounds__(kSmallThreads) lp_small_in_kernel(LpGrid G, const __nv_bfloat16* __restrict__ wb, int dil,
                                                                    const float* __restrict__ d_inv_s,
                                                                    __nv_bfloat16* __restrict__ out) {
    pdl_wait();
    if (G.halt && *G.halt) return;
    __shared__ float W[27 * 3 * 16];
    __shared__ float X[kSmallVox * 27 * 3];
    for (int q = threadIdx.x; q < 27 * 3 * 16; q += kSmallThreads) W[q] = __bfloat162float(wb[q]);
    const float inv_s = *d_inv_s;
    for (int e = threadIdx.x; e < kSmallVox * 27; e += kSmallThreads) {
        const int q = e / 27, tap = e % 27;
        uint32_t v;
        int i, j, k, dx, dy, dz;
        float in[3] = {0.0f, 0.0f, 0.0f};
        if (small_voxel(G, q, v, i, j, k)) {
            tap_off(tap, dx, dy, dz);
            const uint32_t u = small_slot(i + dil * dx, j + dil * dy, k + dil * dz, G.D);
            if (u != 0xFFFFFFFFu) input_channels(G, u, inv_s, in);
        }
        X[3 * e] = in[0];
        X[3 * e + 1] = in[1];
        X[3 * e + 2] = in[2];
    }
    __syncthreads();
    const int co = threadIdx.x & 15, q = threadIdx.x >> 4;
    uint32_t v;
    int i, j, k;
    if (!small_voxel(G, q, v, i, j, k)) return;
    const float* x = X + q * 81;
    float acc = 0.0f;
#pragma unroll 27
    for (int t = 0; t < 81; ++t) acc = fmaf(W[t * 16 + co], x[t], acc);
    out[(size_t)v * 16 + co] = __float2bfloat16_rn(fmaxf(acc, 0.0f));
}

// layers 1, 2 (16 -> 16, ReLU)
__global__ void __launch_bounds__(kSmallThreads) lp_small_mid_kernel(LpGrid G, const __nv_bfloat16* __restrict__ wb, int dil,
                                                                     const __nv_bfloat16* __restrict__ in,
                                                                     __nv_bfloat16* __restrict__ out) {
    pdl_wait();
    if (G.halt && *G.halt) return;
    __shared__ float W[27 * 16 * 16];  // [tap][ci][co]
    __shared__ uint4 X[kSmallVox * 27 * 2];
    for (int q = threadIdx.x; q < 27 * 256; q += kSmallThreads) W[q] = __bfloat162float(wb[q]);
    small_gather16(G, dil, in, X);
    __syncthreads();
    const int co = threadIdx.x & 15, q = threadIdx.x >> 4;
    uint32_t v;
    int i, j, k;
    if (!small_voxel(G, q, v, i, j, k)) return;
    float acc = 0.0f;
    for (int tap = 0; tap < 27; ++tap) {
        float x[16];
        unpack8(X[(q * 27 + tap) * 2], x);
        unpack8(X[(q * 27 + tap) * 2 + 1], x + 8);
        const float* w = W + tap * 256 + co;
#pragma unroll
        for (int ci = 0; ci < 16; ++ci) acc = fmaf(w[ci * 16], x[ci], acc);
    }
    out[(size_t)v * 16 + co] = __float2bfloat16_rn(fmaxf(acc, 0.0f));
}

// layer 3 (16 -> 1) on the fluid cells: thread ci of a voxel sums its input
// channel over the taps, a 16-lane shuffle adds the channels; z = f (raw)
// or z = s (f - f0)
__global__ void __launch_bounds__(kSmallThreads) lp_small_out_kernel(LpGrid G, const __nv_bfloat16* __restrict__ wb, int dil,
                                                                     const __nv_bfloat16* __restrict__ in,
                                                                     const float* __restrict__ d_inv_s,
                                                                     const float* __restrict__ f0, int raw,
                                                                     float* __restrict__ z) {
    pdl_wait();
    if (G.halt && *G.halt) return;
    __shared__ float W[27 * 16];
    __shared__ uint4 X[kSmallVox * 27 * 2];
    for (int q = threadIdx.x; q < 27 * 16; q += kSmallThreads) W[q] = __bfloat162float(wb[q]);
    small_gather16(G, dil, in, X);
    __syncthreads();
    const int ci = threadIdx.x & 15, q = threadIdx.x >> 4;
    uint32_t v = 0;
    int i, j, k;
    const bool ok = small_voxel(G, q, v, i, j, k);
    float acc = 0.0f;
    if (ok) {
        const __nv_bfloat16* xb = reinterpret_cast<const __nv_bfloat16*>(X + q * 54);
        for (int tap = 0; tap < 27; ++tap) acc = fmaf(W[tap * 16 + ci], __bfloat162float(xb[tap * 16 + ci]), acc);
    }
#pragma unroll
    for (int m = 8; m > 0; m >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, m);
    if (ok && ci == 0) {
        float o = 0.0f;
        if (G.type[v] == kFluid) o = raw ? acc : (acc - (f0 ? f0[v] : 0.0f)) * (1.0f / *d_inv_s);
        z[v] = o;
    }
}

static int lp_small_pass(const LpNet& net, const LpGrid& G, const float* d_inv_s, __nv_bfloat16* const* acts,
                         const float* f0, int raw, float* z, uint32_t ntiles, cudaStream_t st) {
    const int g = (int)(ntiles * 512u / kSmallVox);
    // dependent launches: each kernel's launch overlaps its predecessor's tail
    const __nv_bfloat16* a0 = acts[0];
    const __nv_bfloat16* a1 = acts[1];
    const __nv_bfloat16* a2 = acts[2];
    FLIP_CUDA_TRY(pdl_launch(lp_small_in_kernel, g, kSmallThreads, 0, st, G, (const __nv_bfloat16*)(net.wb + kLpWOff[0]),
                             net.dil[0], d_inv_s, acts[0]));
    if (net.tensor_cores) {
        int rc = lp_small_mid_forward_tc(G, net.wb + kLpWOff[1], net.dil[1], a0, acts[1], net.err, ntiles, st);
        if (rc == FLIP_OK) rc = lp_small_mid_forward_tc(G, net.wb + kLpWOff[2], net.dil[2], a1, acts[2], net.err, ntiles, st);
        if (rc != FLIP_OK) return rc;
    } else {
        FLIP_CUDA_TRY(pdl_launch(lp_small_mid_kernel, g, kSmallThreads, 0, st, G,
                                 (const __nv_bfloat16*)(net.wb + kLpWOff[1]), net.dil[1], a0, acts[1]));
        FLIP_CUDA_TRY(pdl_launch(lp_small_mid_kernel, g, kSmallThreads, 0, st, G,
                                 (const __nv_bfloat16*)(net.wb + kLpWOff[2]), net.dil[2], a1, acts[2]));
    }
    FLIP_CUDA_TRY(pdl_launch(lp_small_out_kernel, g, kSmallThreads, 0, st, G, (const __nv_bfloat16*)(net.wb + kLpWOff[3]),
                             net.dil[3], a2, d_inv_s, f0, raw, z));
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int lp_small_bias(const LpNet& net, const LpGrid& G, uint32_t ntiles, const float* d_inv_s, float* f0, cudaStream_t st) {
    LpGrid G0 = G;
    G0.r = nullptr;
    return lp_small_pass(net, G0, d_inv_s, net.actz, nullptr, 1, f0, ntiles, st);
}
int lp_small_forward(const LpNet& net, const LpGrid& G, uint32_t ntiles, const float* d_inv_s, const float* f0, float* z,
                     cudaStream_t st) {
    return lp_small_pass(net, G, d_inv_s, net.act, f0, 0, z, ntiles, st);
}

// --------------------------------------------------------------- backward
// dL/d(layer-2 activations) from dL/dz: G2[u][ci] = relu'(A2[u][ci]) *
// sum_tap W3[tap][ci] * s * gz(u - dil*off); gz is zero off fluid cells
__global__ void __launch_bounds__(512) lp_out_dgrad_kernel(LpGrid G, const __nv_bfloat16* __restrict__ wb, int dil,
                                                           const float* __restrict__ gz, const __nv_bfloat16* __restrict__ a2,
                                                           const float* __restrict__ d_inv_s, float sign,
                                                           float* __restrict__ g2) {
    __shared__ float W[27 * 16];
    for (int i = threadIdx.x; i < 27 * 16; i += 512) W[i] = __bfloat162float(wb[i]);
    __syncthreads();
    const float s = sign / *d_inv_s;
    const uint32_t n = *G.d_nact;
    const int li = threadIdx.x & 7, lj = (threadIdx.x >> 3) & 7, lk = threadIdx.x >> 6;
    for (uint32_t t = blockIdx.x; t < n; t += gridDim.x) {
        const uint32_t key = G.act_tiles[t];
        int ox, oy, oz;
        tile_origin(key, G.D, ox, oy, oz);
        const int i = ox + li, j = oy + lj, k = oz + lk;
        const uint32_t u = (key << 9) | threadIdx.x;
        float acc[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) acc[c] = 0.0f;
        for (int tap = 0; tap < 27; ++tap) {
            int dx, dy, dz;
            tap_off(tap, dx, dy, dz);
            const uint32_t v = active_slot(i - dil * dx, j - dil * dy, k - dil * dz, G);
            if (v == 0xFFFFFFFFu) continue;
            const float g = gz[v];
            if (g == 0.0f) continue;
#pragma unroll
            for (int ci = 0; ci < 16; ++ci) acc[ci] = fmaf(W[tap * 16 + ci], g, acc[ci]);
        }
        float a[16];
        load16(a2, u, a);
        float* out = g2 + (size_t)u * 16;
#pragma unroll
        for (int ci = 0; ci < 16; ++ci) out[ci] = (a[ci] > 0.0f) ? acc[ci] * s : 0.0f;
    }
}

// dL/d(input activations) of a 16 -> 16 layer: Gin[u][ci] = relu'(Ain[u][ci])
// * sum_tap sum_co W[tap][ci][co] * Gout(u - dil*off)[co]
__global__ void __launch_bounds__(512) lp_mid_dgrad_kernel(LpGrid G, const __nv_bfloat16* __restrict__ wb, int dil,
                                                           const float* __restrict__ gout, const __nv_bfloat16* __restrict__ ain,
                                                           float* __restrict__ gin) {
    __shared__ float W[27 * 16 * 16];
    for (int i = threadIdx.x; i < 27 * 256; i += 512) W[i] = __bfloat162float(wb[i]);
    __syncthreads();
    const uint32_t n = *G.d_nact;
    const int li = threadIdx.x & 7, lj = (threadIdx.x >> 3) & 7, lk = threadIdx.x >> 6;
    for (uint32_t t = blockIdx.x; t < n; t += gridDim.x) {
        const uint32_t key = G.act_tiles[t];
        int ox, oy, oz;
        tile_origin(key, G.D, ox, oy, oz);
        const int i = ox + li, j = oy + lj, k = oz + lk;
        const uint32_t u = (key << 9) | threadIdx.x;
        float acc[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) acc[c] = 0.0f;
        for (int tap = 0; tap < 27; ++tap) {
            int dx, dy, dz;
            tap_off(tap, dx, dy, dz);
            const uint32_t v = active_slot(i - dil * dx, j - dil * dy, k - dil * dz, G);
            if (v == 0xFFFFFFFFu) continue;
            const float4* gp = reinterpret_cast<const float4*>(gout + (size_t)v * 16);
            float g[16];
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                float4 f = gp[m];
                g[4 * m] = f.x; g[4 * m + 1] = f.y; g[4 * m + 2] = f.z; g[4 * m + 3] = f.w;
            }
            const float* w = W + tap * 256;
#pragma unroll
            for (int ci = 0; ci < 16; ++ci)
#pragma unroll
                for (int co = 0; co < 16; ++co) acc[ci] = fmaf(w[ci * 16 + co], g[co], acc[ci]);
        }
        float a[16];
        load16(ain, u, a);
        float* out = gin + (size_t)u * 16;
#pragma unroll
        for (int ci = 0; ci < 16; ++ci) out[ci] = (a[ci] > 0.0f) ? acc[ci] : 0.0f;
    }
}

// weight gradient dW[tap][ci][co] += sum_v Gout[v][co] * In(v + dil*off)[ci]
// over the voxels v of the tile list.  Each thread owns one (ci, co) pair and
// a subset of the voxels, and keeps 27 per-tap accumulators.
//   MODE 0: input = the three channels of layer 0 (from r and types)
//   MODE 1: input = 16-channel BF16 activations; COUT 16 (Gout FP32 [slot][16])
//   MODE 2: input = 16-channel activations; COUT 1 (Gout = s*gz, FP32 [slot])
template <int MODE, int CIN, int COUT>
__global__ void __launch_bounds__(512) lp_wgrad_kernel(LpGrid G, int dil, const float* __restrict__ gout,
                                                       const __nv_bfloat16* __restrict__ ain, const float* __restrict__ d_inv_s,
                                                       float sign, const uint32_t* __restrict__ tiles,
                                                       const uint32_t* __restrict__ d_n, float* __restrict__ dw) {
    constexpr int P = CIN * COUT;
    constexpr int S = 512 / P;  // voxel subsets per CTA
    const int pair = threadIdx.x % P, sub = threadIdx.x / P;
    if (sub >= S) return;
    const int ci = pair / COUT, co = pair % COUT;
    const float inv_s = *d_inv_s;
    const float gscale = (MODE == 2) ? sign / inv_s : 1.0f;
    float acc[27];
#pragma unroll
    for (int q = 0; q < 27; ++q) acc[q] = 0.0f;
    const uint32_t n = *d_n;
    for (uint32_t t = blockIdx.x; t < n; t += gridDim.x) {
        const uint32_t key = tiles[t];
        int ox, oy, oz;
        tile_origin(key, G.D, ox, oy, oz);
        for (int vi = sub; vi < 512; vi += S) {
            const uint32_t v = (key << 9) | (uint32_t)vi;
            const float g = (COUT == 1 ? gout[v] : gout[(size_t)v * COUT + co]) * gscale;
            if (g == 0.0f) continue;
            const int i = ox + (vi & 7), j = oy + ((vi >> 3) & 7), k = oz + (vi >> 6);
#pragma unroll
            for (int tap = 0; tap < 27; ++tap) {
                int dx, dy, dz;
                tap_off(tap, dx, dy, dz);
                const uint32_t u = active_slot(i + dil * dx, j + dil * dy, k + dil * dz, G);
                if (u == 0xFFFFFFFFu) continue;
                float x;
                if (MODE == 0) {
                    float in[3];
                    input_channels(G, u, inv_s, in);
                    x = in[ci];
                } else {
                    x = __bfloat162float(ain[(size_t)u * 16 + ci]);
                }
                acc[tap] = fmaf(g, x, acc[tap]);
            }
        }
    }
#pragma unroll
    for (int tap = 0; tap < 27; ++tap)
        if (acc[tap] != 0.0f) atomicAdd(dw + (tap * CIN + ci) * COUT + co, acc[tap]);
}

__global__ void lp_adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                               __nv_bfloat16* __restrict__ wb, int n, float lr, float b1, float b2, float c1, float c2,
                               float eps) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    w[i] = wi;
    wb[i] = __float2bfloat16_rn(wi);
}

__global__ void lp_to_bf16_kernel(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) wb[i] = __float2bfloat16_rn(w[i]);
}

// ------------------------------------------------------------ launchers
// the three hidden layers into acts[0..2]
static int lp_hidden(const LpNet& net, const LpGrid& G, const float* d_inv_s, __nv_bfloat16* const* acts, int grid,
                     cudaStream_t st) {
    lp_in_kernel<<<grid, 512, 0, st>>>(G, net.wb + kLpWOff[0], net.dil[0], d_inv_s, acts[0]);
    if (net.tensor_cores) {
        int rc = lp_mid_forward_tc(G, net.wb + kLpWOff[1], net.dil[1], acts[0], acts[1], net.err, net.sms, st);
        if (rc == FLIP_OK) rc = lp_mid_forward_tc(G, net.wb + kLpWOff[2], net.dil[2], acts[1], acts[2], net.err, net.sms, st);
        if (rc != FLIP_OK) return rc;
    } else {
        lp_mid_kernel<<<grid, 512, 0, st>>>(G, net.wb + kLpWOff[1], net.dil[1], acts[0], acts[1]);
        lp_mid_kernel<<<grid, 512, 0, st>>>(G, net.wb + kLpWOff[2], net.dil[2], acts[1], acts[2]);
    }
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int lp_bias_dev(const LpNet& net, const LpGrid& G, const float* d_inv_s, float* f0, int grid, cudaStream_t st) {
    LpGrid G0 = G;
    G0.r = nullptr;
    int rc = lp_hidden(net, G0, d_inv_s, net.actz, grid, st);
    if (rc != FLIP_OK) return rc;
    lp_out_kernel<<<grid, 512, 0, st>>>(G0, net.wb + kLpWOff[3], net.dil[3], net.actz[2], d_inv_s, nullptr, 1, f0);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int lp_forward_dev(const LpNet& net, const LpGrid& G, const float* d_inv_s, const float* f0, float* z, int grid,
                   cudaStream_t st) {
    int rc = lp_hidden(net, G, d_inv_s, net.act, grid, st);
    if (rc != FLIP_OK) return rc;
    lp_out_kernel<<<grid, 512, 0, st>>>(G, net.wb + kLpWOff[3], net.dil[3], net.act[2], d_inv_s, f0, 0, z);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

// one backward pass through the activations acts, dL/d(output) = sign * s * gz
static int lp_backward_path(LpNet& net, const LpGrid& G, const float* d_inv_s, const float* gz,
                            __nv_bfloat16* const* acts, float sign, int grid, cudaStream_t st) {
    // layer 3 (16 -> 1)
    if (net.tensor_cores) {
        const int rc = lp_out_wgrad_tc(G, net.dil[3], gz, acts[2], d_inv_s, sign, net.g + kLpWOff[3], net.err, net.sms, st);
        if (rc != FLIP_OK) return rc;
    } else {
        lp_wgrad_kernel<2, 16, 1><<<grid, 512, 0, st>>>(G, net.dil[3], gz, acts[2], d_inv_s, sign, G.out_tiles, G.d_nout,
                                                        net.g + kLpWOff[3]);
    }
    lp_out_dgrad_kernel<<<grid, 512, 0, st>>>(G, net.wb + kLpWOff[3], net.dil[3], gz, acts[2], d_inv_s, sign, net.gact);
    if (net.tensor_cores) {
        // layer 2 (16 -> 16): Gout = gact (wrt act[2]), input act[1]; then layer 1
        int rc = lp_mid_wgrad_tc(G, net.dil[2], net.gact, acts[1], net.g + kLpWOff[2], net.err, net.sms, st);
        if (rc == FLIP_OK)
            rc = lp_mid_dgrad_tc(G, net.wb + kLpWOff[2], net.dil[2], net.gact, acts[1], net.gact2, net.err, net.sms, st);
        if (rc == FLIP_OK) rc = lp_mid_wgrad_tc(G, net.dil[1], net.gact2, acts[0], net.g + kLpWOff[1], net.err, net.sms, st);
        if (rc == FLIP_OK)
            rc = lp_mid_dgrad_tc(G, net.wb + kLpWOff[1], net.dil[1], net.gact2, acts[0], net.gact, net.err, net.sms, st);
        if (rc != FLIP_OK) return rc;
    } else {
        // layer 2 (16 -> 16): Gout = gact (wrt act[2]), input act[1]
        lp_wgrad_kernel<1, 16, 16><<<grid, 512, 0, st>>>(G, net.dil[2], net.gact, acts[1], d_inv_s, 1.0f, G.act_tiles,
                                                         G.d_nact, net.g + kLpWOff[2]);
        lp_mid_dgrad_kernel<<<grid, 512, 0, st>>>(G, net.wb + kLpWOff[2], net.dil[2], net.gact, acts[1], net.gact2);
        // layer 1: Gout = gact2 (wrt act[1]), input act[0]
        lp_wgrad_kernel<1, 16, 16><<<grid, 512, 0, st>>>(G, net.dil[1], net.gact2, acts[0], d_inv_s, 1.0f, G.act_tiles,
                                                         G.d_nact, net.g + kLpWOff[1]);
        lp_mid_dgrad_kernel<<<grid, 512, 0, st>>>(G, net.wb + kLpWOff[1], net.dil[1], net.gact2, acts[0], net.gact);
    }
    // layer 0: Gout = gact (wrt act[0]), input = the three channels
    if (net.tensor_cores) {
        const int rc = lp_in_wgrad_tc(G, net.dil[0], net.gact, d_inv_s, net.g + kLpWOff[0], net.err, net.sms, st);
        if (rc != FLIP_OK) return rc;
    } else {
        lp_wgrad_kernel<0, 3, 16><<<grid, 512, 0, st>>>(G, net.dil[0], net.gact, nullptr, d_inv_s, 1.0f, G.act_tiles,
                                                        G.d_nact, net.g + kLpWOff[0]);
    }
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int lp_backward_dev(LpNet& net, const LpGrid& G, const float* d_inv_s, const float* gz, int grid, cudaStream_t st) {
    int rc = lp_backward_path(net, G, d_inv_s, gz, net.act, 1.0f, grid, st);
    if (rc != FLIP_OK) return rc;
    LpGrid G0 = G;
    G0.r = nullptr;  // the zero-residual pass enters with a minus sign
    return lp_backward_path(net, G0, d_inv_s, gz, net.actz, -1.0f, grid, st);
}

// m = N(r) + D^-1 r at a fluid cell from its slot
__device__ __forceinline__ float lp_m(const float* __restrict__ z, const LpGrid& G, uint32_t u, uint8_t c) {
    const float d = (float)(c & 7u);
    return d > 0.0f ? z[u] + G.r[u] / d : z[u];
}

// A m - r on fluid cells; sums m.Am, m.r, e.r
__global__ void __launch_bounds__(512) lp_anorm_kernel(LpGrid G, const float* __restrict__ z, const float* __restrict__ ev,
                                                       float* __restrict__ wbuf, double* __restrict__ sums) {
    __shared__ double sh[32];
    const uint32_t n = *G.d_nout;
    const int li = threadIdx.x & 7, lj = (threadIdx.x >> 3) & 7, lk = threadIdx.x >> 6;
    double mam = 0.0, mr = 0.0, er = 0.0;
    for (uint32_t t = blockIdx.x; t < n; t += gridDim.x) {
        const uint32_t key = G.out_tiles[t];
        int ox, oy, oz;
        tile_origin(key, G.D, ox, oy, oz);
        const uint32_t v = (key << 9) | threadIdx.x;
        const uint8_t c = G.cell[v];
        float wv = 0.0f;
        if (c & 0x80u) {
            const int i = ox + li, j = oy + lj, k = oz + lk;
            const float m = lp_m(z, G, v, c);
            const int oi[6] = {-1, 1, 0, 0, 0, 0}, oj[6] = {0, 0, -1, 1, 0, 0}, ok[6] = {0, 0, 0, 0, -1, 1};
            float sum = 0.0f;
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                const int a = i + oi[q], b = j + oj[q], cc = k + ok[q];
                if (a < 0 || b < 0 || cc < 0 || a >= G.D.nx || b >= G.D.ny || cc >= G.D.nz) continue;
                const uint32_t u = lslot(a, b, cc, G.D);
                const uint8_t cu = G.cell[u];
                if (cu & 0x80u) sum += lp_m(z, G, u, cu);
            }
            const float am = fmaf((float)(c & 7u), m, -sum);
            const float rv = G.r[v];
            wv = am - rv;
            mam += (double)m * (double)am;
            mr += (double)m * (double)rv;
            er += (double)ev[v] * (double)rv;
        }
        wbuf[v] = wv;
    }
    const double a = block_sum_f64<512>(mam, sh);
    const double b = block_sum_f64<512>(mr, sh);
    const double e = block_sum_f64<512>(er, sh);
    if (threadIdx.x == 0) {
        if (a != 0.0) atomicAdd(sums, a);
        if (b != 0.0) atomicAdd(sums + 1, b);
        if (e != 0.0) atomicAdd(sums + 2, e);
    }
}

__global__ void __launch_bounds__(512) lp_anorm_gz_kernel(LpGrid G, const float* __restrict__ wbuf,
                                                          const double* __restrict__ sums, float* __restrict__ gz) {
    const double er = sums[2];
    const float scale = er > 0.0 ? (float)(2.0 / er) : 0.0f;
    const uint32_t n = *G.d_nact;
    for (uint32_t t = blockIdx.x; t < n; t += gridDim.x) {
        const uint32_t v = (G.act_tiles[t] << 9) | threadIdx.x;
        gz[v] = (G.cell[v] & 0x80u) ? scale * wbuf[v] : 0.0f;
    }
}

int lp_loss_grad(const LpGrid& G, const float* z, const float* ev, float* wbuf, float* gz, double* d_sums, int grid,
                 cudaStream_t st) {
    lp_anorm_kernel<<<grid, 512, 0, st>>>(G, z, ev, wbuf, d_sums);
    lp_anorm_gz_kernel<<<grid, 512, 0, st>>>(G, wbuf, d_sums, gz);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

// counter-based normal numbers: splitmix64 of (seed, slot), Box-Muller
__device__ __forceinline__ uint64_t lp_mix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
__global__ void __launch_bounds__(512) lp_noise_kernel(LpGrid G, uint64_t seed, float* __restrict__ ev) {
    const uint32_t n = *G.d_nout;
    for (uint32_t t = blockIdx.x; t < n; t += gridDim.x) {
        const uint32_t v = (G.out_tiles[t] << 9) | threadIdx.x;
        float e = 0.0f;
        if (G.cell[v] & 0x80u) {
            const uint64_t h = lp_mix(seed * 0x100000001B3ull + v);
            const float u1 = ((float)(h >> 40) + 0.5f) * (1.0f / 16777216.0f);
            const float u2 = (float)((h >> 16) & 0xFFFFFFull) * (1.0f / 16777216.0f);
            e = sqrtf(-2.0f * logf(u1)) * cosf(6.283185307f * u2);
        }
        ev[v] = e;
    }
}
__global__ void __launch_bounds__(512) lp_apply_A_kernel(LpGrid G, const float* __restrict__ x, float* __restrict__ y) {
    const uint32_t n = *G.d_nout;
    const int li = threadIdx.x & 7, lj = (threadIdx.x >> 3) & 7, lk = threadIdx.x >> 6;
    for (uint32_t t = blockIdx.x; t < n; t += gridDim.x) {
        const uint32_t key = G.out_tiles[t];
        int ox, oy, oz;
        tile_origin(key, G.D, ox, oy, oz);
        const uint32_t v = (key << 9) | threadIdx.x;
        const uint8_t c = G.cell[v];
        float out = 0.0f;
        if (c & 0x80u) {
            const int i = ox + li, j = oy + lj, k = oz + lk;
            const int oi[6] = {-1, 1, 0, 0, 0, 0}, oj[6] = {0, 0, -1, 1, 0, 0}, ok[6] = {0, 0, 0, 0, -1, 1};
            float sum = 0.0f;
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                const int a = i + oi[q], b = j + oj[q], cc = k + ok[q];
                if (a < 0 || b < 0 || cc < 0 || a >= G.D.nx || b >= G.D.ny || cc >= G.D.nz) continue;
                const uint32_t u = lslot(a, b, cc, G.D);
                if (G.cell[u] & 0x80u) sum += x[u];
            }
            out = fmaf((float)(c & 7u), x[v], -sum);
        }
        y[v] = out;
    }
}
int lp_noise_sample(const LpGrid& G, uint64_t seed, float* ev, float* r, int grid, cudaStream_t st) {
    lp_noise_kernel<<<grid, 512, 0, st>>>(G, seed, ev);
    lp_apply_A_kernel<<<grid, 512, 0, st>>>(G, ev, r);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

__global__ void __launch_bounds__(512) lp_solution_kernel(LpGrid G, const double* __restrict__ x, const float* __restrict__ xg,
                                                          const float* __restrict__ xs, float* __restrict__ out) {
    const uint32_t n = *G.d_nout;
    for (uint32_t t = blockIdx.x; t < n; t += gridDim.x) {
        const uint32_t v = (G.out_tiles[t] << 9) | threadIdx.x;
        float o = 0.0f;
        if (G.cell[v] & 0x80u) {
            const double xv = x[v] + (double)xg[v];
            o = xs ? (float)((double)xs[v] - xv) : (float)xv;
        }
        out[v] = o;
    }
}
int lp_store_solution(const LpGrid& G, const double* x, const float* xg, float* xs, int grid, cudaStream_t st) {
    lp_solution_kernel<<<grid, 512, 0, st>>>(G, x, xg, nullptr, xs);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int lp_error_from_solution(const LpGrid& G, const double* x, const float* xg, const float* xs, float* ev, int grid,
                           cudaStream_t st) {
    lp_solution_kernel<<<grid, 512, 0, st>>>(G, x, xg, xs, ev);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

// sum of r^2 over the fluid cells of the output tiles into *acc (zeroed by the caller)
__global__ void __launch_bounds__(512) lp_rr_kernel(LpGrid G, double* __restrict__ acc) {
    __shared__ double sh[32];
    const uint32_t n = *G.d_nout;
    double a = 0.0;
    for (uint32_t t = blockIdx.x; t < n; t += gridDim.x) {
        const uint32_t v = (G.out_tiles[t] << 9) | threadIdx.x;
        if (G.type[v] == kFluid) a += (double)G.r[v] * (double)G.r[v];
    }
    double r = block_sum_f64<512>(a, sh);
    if (threadIdx.x == 0 && r != 0.0) atomicAdd(acc, r);
}
__global__ void lp_inv_s_kernel(const double* __restrict__ acc, const double* __restrict__ nfluid, float* __restrict__ inv_s) {
    const double rr = *acc, nf = fmax(*nfluid, 1.0);
    *inv_s = rr > 0.0 ? (float)(1.0 / sqrt(rr / nf)) : 1.0f;
}
int lp_input_scale(const LpGrid& G, double* d_acc, const double* d_nfluid, float* d_inv_s, int grid, cudaStream_t st) {
    FLIP_CUDA_TRY(cudaMemsetAsync(d_acc, 0, sizeof(double), st));
    lp_rr_kernel<<<grid, 512, 0, st>>>(G, d_acc);
    lp_inv_s_kernel<<<1, 1, 0, st>>>(d_acc, d_nfluid, d_inv_s);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int lp_adam(LpNet& net, float lr, cudaStream_t st) {
    net.adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.0f / (1.0f - powf(b1, (float)net.adam_t)), c2 = 1.0f / (1.0f - powf(b2, (float)net.adam_t));
    lp_adam_kernel<<<(kLpNumW + 255) / 256, 256, 0, st>>>(net.w, net.g, net.m, net.v, net.wb, kLpNumW, lr, b1, b2, c1, c2, eps);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int lp_sync_bf16(LpNet& net, cudaStream_t st) {
    lp_to_bf16_kernel<<<(kLpNumW + 255) / 256, 256, 0, st>>>(net.w, net.wb, kLpNumW);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

}  // namespace flip
