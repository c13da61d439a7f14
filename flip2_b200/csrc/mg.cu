// mg.cu -- V-cycle kernels of the multilevel learned preconditioner (mg.cuh).
//
// Every level is tile-blocked like the solver's grid (slot = tile * 512 +
// (i & 7) + 8 (j & 7) + 64 (k & 7)).  Per level the hierarchy kernels
// (coarse types, cell codes) walk every slot; the two smoothing kernels walk
// the level's tile list and stage each tile with a 2-cell halo in shared
// memory (see "smoothing" below); the coarsest level also has a one-CTA
// Jacobi-PCG (training targets, and the comparison without the network).
// Non-fluid cells carry 0 in every vector, so the 7-point operator needs only
// the fluid bit and the non-solid neighbour count of the PCG cell code.
#include "common.cuh"
#include "mg.cuh"

namespace flip {

__device__ __forceinline__ uint32_t mg_slot(int i, int j, int k, const NatDims& D) {
    uint32_t t = (uint32_t)((i >> 3) + D.tx * ((j >> 3) + D.ty * (k >> 3)));
    return (t << 9) | (uint32_t)((i & 7) | ((j & 7) << 3) | ((k & 7) << 6));
}
__device__ __forceinline__ void mg_cell_of(uint32_t key, int tid, const NatDims& D, int& i, int& j, int& k) {
    i = 8 * (int)(key % D.tx) + (tid & 7);
    j = 8 * (int)((key / D.tx) % D.ty) + ((tid >> 3) & 7);
    k = 8 * (int)(key / (D.tx * D.ty)) + (tid >> 6);
}
__device__ __forceinline__ bool mg_in(int i, int j, int k, const NatDims& D) {
    return i >= 0 && j >= 0 && k >= 0 && i < D.nx && j < D.ny && k < D.nz;
}
__device__ __forceinline__ float mg_dinv(uint8_t c) {
    const uint32_t d = c & 7u;
    return d ? 1.0f / (float)d : 0.0f;
}
// sum over the fluid neighbours of (i, j, k) of val(slot)
template <class F>
__device__ __forceinline__ float mg_nb_sum(int i, int j, int k, const NatDims& D, const uint8_t* __restrict__ cell, F val) {
    const int oi[6] = {-1, 1, 0, 0, 0, 0}, oj[6] = {0, 0, -1, 1, 0, 0}, ok[6] = {0, 0, 0, 0, -1, 1};
    float s = 0.0f;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const int a = i + oi[q], b = j + oj[q], c = k + ok[q];
        if (!mg_in(a, b, c, D)) continue;
        const uint32_t u = mg_slot(a, b, c, D);
        if (cell[u] & kCellFluid) s += val(u);
    }
    return s;
}
__device__ __forceinline__ bool mg_halted(const int* halt) { return halt && *halt; }

// ------------------------------------------------------------ hierarchy
// coarse type from the 8 children: air if any child is air, else fluid if any
// is fluid, else solid; cells past the level's extent are solid
__global__ void __launch_bounds__(512) mg_coarsen_kernel(MgLevel F, MgLevel C, const int* halt) {
    if (mg_halted(halt)) return;
    const uint32_t n = C.ntiles * 512u;
    for (uint32_t s = blockIdx.x * 512u + threadIdx.x; s < n; s += gridDim.x * 512u) {
        int I, J, K;
        mg_cell_of(s >> 9, (int)(s & 511u), C.D, I, J, K);
        uint8_t t = kSolid;
        if (I < C.ex && J < C.ey && K < C.ez) {
            bool air = false, fluid = false;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int i = 2 * I + (c & 1), j = 2 * J + ((c >> 1) & 1), k = 2 * K + (c >> 2);
                if (i >= F.ex || j >= F.ey || k >= F.ez) continue;  // solid
                const uint8_t ft = F.type[mg_slot(i, j, k, F.D)];
                air |= ft == kAir;
                fluid |= ft == kFluid;
            }
            t = air ? kAir : (fluid ? kFluid : kSolid);
        }
        C.type[s] = t;
    }
}
// PCG cell codes of a coarse level: fluid bit and the non-solid neighbour count
__global__ void __launch_bounds__(512) mg_codes_kernel(MgLevel C, const int* halt) {
    if (mg_halted(halt)) return;
    const uint32_t n = C.ntiles * 512u;
    const int oi[6] = {-1, 1, 0, 0, 0, 0}, oj[6] = {0, 0, -1, 1, 0, 0}, ok[6] = {0, 0, 0, 0, -1, 1};
    for (uint32_t s = blockIdx.x * 512u + threadIdx.x; s < n; s += gridDim.x * 512u) {
        uint8_t code = 0;
        if (C.type[s] == kFluid) {
            int i, j, k;
            mg_cell_of(s >> 9, (int)(s & 511u), C.D, i, j, k);
            uint32_t d = 0;
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                const int a = i + oi[q], b = j + oj[q], c = k + ok[q];
                if (mg_in(a, b, c, C.D) && C.type[mg_slot(a, b, c, C.D)] != kSolid) ++d;
            }
            code = (uint8_t)(kCellFluid | d);
        }
        C.cell[s] = code;
    }
}

// ------------------------------------------------------------ smoothing
// The V-cycle's smoothing runs as two kernels per level.  Each CTA stages a
// box of its tile and a 2-cell halo in shared memory: 16 cells wide in x
// (x = -4 .. 11, so that every row is four 16-byte quads of the tile
// layout: x 4..7 of the left tile, the tile's two quads, x 0..3 of the right
// tile) and 12 in y and z (-2 .. 9).  The first sweep is evaluated on whole
// quads of the rows y, z = -1 .. 8 (only x = -1 .. 8 of them is used), the
// second sweep (or the residual) on the tile's 128 quads.  A thread handles
// four cells: float4 global loads and stores, float4 shared rows.  Vectors
// are zero off the fluid cells, so a neighbour sum needs no tests; 1/d comes
// from a shared table.  Five CTAs per SM keep tiles in flight: one CTA's
// loads overlap the others' barriers and arithmetic.
constexpr int kMgThreads = 256;
constexpr int kBX = 16, kBY = 12, kBZ = 12;
constexpr int kBoxQ = kBX * kBY * kBZ / 4;      // 576 quads in the box
constexpr int kBoxF = kBX * kBY * kBZ;          // 2304 cells
constexpr int kSw1Q = 4 * 10 * 10;              // 400 quads of the first sweep
constexpr int kT1F = kBX * 10 * 10;             // its output box, 1600 cells
constexpr int kQPer = (kBoxQ + kMgThreads - 1) / kMgThreads;  // 3

// Two FP64 sums over the grid of a level kernel: per-CTA sums into
// partials[q * gridDim.x + CTA], then the last CTA to arrive adds the
// partials in CTA order (deterministic for a given grid), resets the ticket
// and returns true with the totals in thread 0's out.
__device__ __forceinline__ bool mg_last_cta_sum2(double v0, double v1, double* partials, unsigned int* ticket,
                                                 double (&out)[2]) {
    __shared__ double sh[32];
    __shared__ bool s_last;
    const double v[2] = {v0, v1};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const double s = block_sum_f64<kMgThreads>(v[q], sh);
        if (threadIdx.x == 0) partials[q * gridDim.x + blockIdx.x] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        double a = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += kMgThreads) a += ((volatile double*)partials)[q * gridDim.x + b];
        out[q] = block_sum_f64<kMgThreads>(a, sh);
    }
    if (threadIdx.x == 0) *ticket = 0u;
    return true;
}

// box quad q -> (neighbour tile offset + 1 per axis, local slot of its first
// cell), packed as local | (qx + 1) << 9 | (qy + 1) << 11 | (qz + 1) << 13; -1 past the box
__device__ __forceinline__ int mg_quad_map(int q) {
    if (q >= kBoxQ) return -1;
    const int seg = q & 3, row = q >> 2;
    const int y = row % kBY - 2, z = row / kBY - 2;
    const int qx = seg == 0 ? -1 : (seg == 3 ? 1 : 0);
    const int lx = seg == 0 ? 4 : (seg == 3 ? 0 : 4 * (seg - 1));
    const int qy = (y + 8) / 8 - 1, qz = (z + 8) / 8 - 1;
    const int local = lx | ((y - 8 * qy) << 3) | ((z - 8 * qz) << 6);
    return local | ((qx + 1) << 9) | ((qy + 1) << 11) | ((qz + 1) << 13);
}
// slot of a mapped quad's first cell around the tile at tile coordinates
// (tx, ty, tz), or UINT32_MAX outside the grid; the cell's (i, j, k) out
__device__ __forceinline__ uint32_t mg_quad_slot(int map, int tx, int ty, int tz, const NatDims& D, int& i, int& j, int& k) {
    const int ntx = tx + ((map >> 9) & 3) - 1, nty = ty + ((map >> 11) & 3) - 1, ntz = tz + ((map >> 13) & 3) - 1;
    i = 8 * ntx + (map & 7);
    j = 8 * nty + ((map >> 3) & 7);
    k = 8 * ntz + ((map >> 6) & 7);
    if (map < 0 || ntx < 0 || nty < 0 || ntz < 0 || ntx >= D.tx || nty >= D.ty || ntz >= D.tz) return 0xFFFFFFFFu;
    return ((uint32_t)(ntx + D.tx * (nty + D.ty * ntz)) << 9) | (uint32_t)(map & 511);
}
__device__ __forceinline__ void mg_tile_xyz(uint32_t key, const NatDims& D, int& tx, int& ty, int& tz) {
    const uint32_t tyz = key / (uint32_t)D.tx;
    tx = (int)(key - tyz * (uint32_t)D.tx);
    ty = (int)(tyz % (uint32_t)D.ty);
    tz = (int)(tyz / (uint32_t)D.ty);
}
__device__ __forceinline__ void mg_inv_table(float* inv) {
    if (threadIdx.x < 8) inv[threadIdx.x] = threadIdx.x ? 1.0f / (float)threadIdx.x : 0.0f;
}
__device__ __forceinline__ float f4(const float4& v, int m) { return m == 0 ? v.x : (m == 1 ? v.y : (m == 2 ? v.z : v.w)); }
__device__ __forceinline__ void f4set(float4& v, int m, float x) {
    if (m == 0) v.x = x; else if (m == 1) v.y = x; else if (m == 2) v.z = x; else v.w = x;
}
// one damped Jacobi sweep of a quad: out = u + w D^-1 (r - (d u - nb)) on its
// fluid cells (0 elsewhere); nb: sums of the six neighbours per cell
__device__ __forceinline__ float4 mg_quad_sweep(uint32_t c4, const float4& u, const float4& r, const float4& nb,
                                                const float* inv) {
    float4 o;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const uint32_t c = (c4 >> (8 * m)) & 0xFFu;
        const float d = (float)(c & 7u);
        const float um = f4(u, m);
        f4set(o, m, (c & kCellFluid) ? um + kMgOmega * inv[c & 7u] * (f4(r, m) - (d * um - f4(nb, m))) : 0.0f);
    }
    return o;
}
// neighbour sums of the quad at float index b of a box of row stride SY and
// plane stride SZ (rows of 16 floats), c its own values, l and r the cells
// left of its first and right of its last.  The x neighbours come from the
// neighbouring lanes rather than from scalar shared loads, which hit their
// banks four times over:
//   mg_quad_nb_row: the four quads of a row sit in four consecutive active
//     lanes (qd = the quad's place in its row; the first sweep's layout);
//   mg_quad_nb_pair: quads 1 and 2 of a row sit in lanes 2k, 2k + 1 of a full
//     warp (the second sweep's layout); the outer neighbour still comes from
//     shared memory.
template <int SY, int SZ>
__device__ __forceinline__ float4 mg_quad_nb_yz(const float* v, int b, const float4& c, float l, float r) {
    const float4 ym = *reinterpret_cast<const float4*>(v + b - SY), yp = *reinterpret_cast<const float4*>(v + b + SY);
    const float4 zm = *reinterpret_cast<const float4*>(v + b - SZ), zp = *reinterpret_cast<const float4*>(v + b + SZ);
    float4 s;
    s.x = ((l + c.y) + (ym.x + yp.x)) + (zm.x + zp.x);
    s.y = ((c.x + c.z) + (ym.y + yp.y)) + (zm.y + zp.y);
    s.z = ((c.y + c.w) + (ym.z + yp.z)) + (zm.z + zp.z);
    s.w = ((c.z + r) + (ym.w + yp.w)) + (zm.w + zp.w);
    return s;
}
template <int SY, int SZ>
__device__ __forceinline__ float4 mg_quad_nb_row(const float* v, int b, int qd, const float4& c) {
    const unsigned m = __activemask();
    const float l = __shfl_up_sync(m, c.w, 1), r = __shfl_down_sync(m, c.x, 1);
    return mg_quad_nb_yz<SY, SZ>(v, b, c, qd > 0 ? l : 0.0f, qd < 3 ? r : 0.0f);
}
template <int SY, int SZ>
__device__ __forceinline__ float4 mg_quad_nb_pair(const float* v, int b, int half, const float4& c) {
    const float got = __shfl_xor_sync(0xffffffffu, half ? c.x : c.w, 1);
    const float outer = v[b + (half ? 4 : -1)];
    return mg_quad_nb_yz<SY, SZ>(v, b, c, half ? got : outer, half ? outer : got);
}

// pre-smoothing and restriction of level F into C:
//   t1 = w D^-1 r, t = t1 + w D^-1 (r - A t1) (kept in F.t),
//   C.r[parent] = 1/2 sum over the 8 children of r - A t (fluid parents; the
//   parents of a tile are all written by it, and parents of tiles off the
//   list are never fluid)
template <bool SCALE = false>
__global__ void __launch_bounds__(kMgThreads, 5) mg_down_kernel(MgLevel F, MgLevel C, const int* halt, MgScale sc) {
    pdl_wait();
    if (mg_halted(halt)) return;
    // SCALE (C the coarsest level): the sum of C.r^2 and the count over the
    // fluid parents this CTA writes, then *sc.inv_s as mg_scale_kernel sets it
    __shared__ double acc[SCALE ? 2 * 64 : 1];
    if (SCALE && threadIdx.x < 64) acc[2 * threadIdx.x] = acc[2 * threadIdx.x + 1] = 0.0;
    __shared__ uint32_t cb[kBoxQ];                  // four codes per quad
    __shared__ __align__(16) float rb[kBoxF];
    __shared__ __align__(16) float ub[kBoxF];       // t1 = w D^-1 r
    __shared__ __align__(16) float tb[kT1F];        // first sweep
    __shared__ float S[256];                        // x-pair sums of the residual
    __shared__ float inv[8];
    mg_inv_table(inv);
    const int tid = threadIdx.x;
    int map[kQPer];
#pragma unroll
    for (int m = 0; m < kQPer; ++m) map[m] = mg_quad_map(tid + m * kMgThreads);
    const uint32_t n = *F.d_ntiles;
    uint32_t pc[kQPer];
    float4 pr[kQPer];
    auto fetch = [&](uint32_t tt) {
        int tx, ty, tz, i, j, k;
        mg_tile_xyz(F.tiles[tt], F.D, tx, ty, tz);
#pragma unroll
        for (int m = 0; m < kQPer; ++m) {
            const uint32_t sl = mg_quad_slot(map[m], tx, ty, tz, F.D, i, j, k);
            pc[m] = 0u;
            pr[m] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (sl != 0xFFFFFFFFu) {
                pc[m] = *reinterpret_cast<const uint32_t*>(F.cell + sl);
                pr[m] = *reinterpret_cast<const float4*>(F.r + sl);
            }
        }
    };
    __syncthreads();  // the 1/d table
    for (uint32_t tt = blockIdx.x; tt < n; tt += gridDim.x) {
        const uint32_t key = F.tiles[tt];
        fetch(tt);
#pragma unroll
        for (int m = 0; m < kQPer; ++m) {
            const int q = tid + m * kMgThreads;
            if (q < kBoxQ) {
                const uint32_t c4 = pc[m];
                float4 r, u;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const uint32_t c = (c4 >> (8 * e)) & 0xFFu;
                    const float rv = (c & kCellFluid) ? f4(pr[m], e) : 0.0f;
                    f4set(r, e, rv);
                    f4set(u, e, kMgOmega * inv[c & 7u] * rv);
                }
                cb[q] = c4;
                *reinterpret_cast<float4*>(rb + 4 * q) = r;
                *reinterpret_cast<float4*>(ub + 4 * q) = u;
            }
        }
        __syncthreads();
        for (int w = tid; w < kSw1Q; w += kMgThreads) {
            const int qd = w & 3, row = w >> 2;
            const int by = row % 10 + 1, bz = row / 10 + 1;
            const int b = 4 * qd + kBX * (by + kBY * bz);
            const float4 uc = *reinterpret_cast<const float4*>(ub + b);
            const float4 o = mg_quad_sweep(cb[b >> 2], uc, *reinterpret_cast<const float4*>(rb + b),
                                           mg_quad_nb_row<kBX, kBX * kBY>(ub, b, qd, uc), inv);
            *reinterpret_cast<float4*>(tb + 4 * qd + kBX * (row % 10 + 10 * (row / 10))) = o;
        }
        __syncthreads();
        if (tid < 128) {
            const int half = tid & 1, row = tid >> 1, ly = row & 7, lz = row >> 3;
            const int qd = 1 + half;
            const int b = 4 * qd + kBX * ((ly + 2) + kBY * (lz + 2));
            const int t = 4 * qd + kBX * ((ly + 1) + 10 * (lz + 1));
            const uint32_t c4 = cb[b >> 2];
            const float4 tv = *reinterpret_cast<const float4*>(tb + t), r = *reinterpret_cast<const float4*>(rb + b);
            const float4 nb = mg_quad_nb_pair<kBX, kBX * 10>(tb, t, half, tv);
            float res[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const uint32_t c = (c4 >> (8 * m)) & 0xFFu;
                res[m] = (c & kCellFluid) ? f4(r, m) - ((float)(c & 7u) * f4(tv, m) - f4(nb, m)) : 0.0f;
            }
            *reinterpret_cast<float4*>(F.t + ((key << 9) | (uint32_t)(4 * half + 8 * ly + 64 * lz))) = tv;
            S[(2 * half) + 4 * (ly + 8 * lz)] = res[0] + res[1];
            S[(2 * half + 1) + 4 * (ly + 8 * lz)] = res[2] + res[3];
        }
        __syncthreads();
        if (tid < 64) {  // parent (pi, pj, pk) of the tile's 4^3 parents
            int tx, ty, tz;
            mg_tile_xyz(key, F.D, tx, ty, tz);
            const int pi = tid & 3, pj = (tid >> 2) & 3, pk = tid >> 4;
            const int s0 = pi + 4 * (2 * pj + 8 * 2 * pk);
            const float sum = (S[s0] + S[s0 + 4]) + (S[s0 + 32] + S[s0 + 36]);
            const uint32_t p = mg_slot(4 * tx + pi, 4 * ty + pj, 4 * tz + pk, C.D);
            const bool fl = (C.cell[p] & kCellFluid) != 0;
            const float v = fl ? 0.5f * sum : 0.0f;
            C.r[p] = v;
            if (SCALE && fl) {
                acc[2 * tid] += (double)v * (double)v;
                acc[2 * tid + 1] += 1.0;
            }
        }
        __syncthreads();
    }
    if (SCALE) {
        double out[2];
        const bool last = mg_last_cta_sum2(tid < 64 ? acc[2 * tid] : 0.0, tid < 64 ? acc[2 * tid + 1] : 0.0,
                                           sc.partials, sc.ticket, out);
        if (last && tid == 0) *sc.inv_s = out[0] > 0.0 ? (float)(1.0 / sqrt(out[0] / fmax(out[1], 1.0))) : 1.0f;
    }
}

// two damped Jacobi sweeps from a start vector u: t2 = u + w D^-1 (r - A u),
// L.z = t2 + w D^-1 (r - A t2).  MODE 0: u = L.t + C.z[parent] (prolongation
// of the coarse correction; post-smoothing); MODE 1: u = zn + D^-1 r (the
// coarsest level with the network output zn); MODE 2: u = w D^-1 r (the
// coarsest level without the network); MODE 3: u = zn (the coarsest level
// after a CG solve into zn).  DOT (MODE 0 on level 0): FCG's dot products
// of the z it writes (MgDot), reduced by the last CTA.
template <int MODE, bool DOT = false>
__global__ void __launch_bounds__(kMgThreads, 5) mg_sweeps_kernel(MgLevel L, MgLevel C, const float* __restrict__ zn,
                                                                  const int* halt, MgDot dot) {
    pdl_wait();
    if (mg_halted(halt)) return;
    __shared__ uint32_t cb[kBoxQ];
    __shared__ __align__(16) float rb[kBoxF];
    __shared__ __align__(16) float ub[kBoxF];
    __shared__ __align__(16) float tb[kT1F];
    __shared__ float inv[8];
    __shared__ double acc[DOT ? 2 * 128 : 1];  // r.z, z.q of each storing thread
    mg_inv_table(inv);
    const int tid = threadIdx.x;
    if (DOT && tid < 128) acc[2 * tid] = acc[2 * tid + 1] = 0.0;
    int map[kQPer];
#pragma unroll
    for (int m = 0; m < kQPer; ++m) map[m] = mg_quad_map(tid + m * kMgThreads);
    const uint32_t n = *L.d_ntiles;
    uint32_t pc[kQPer];
    float4 pr[kQPer], pu[kQPer];
    float2 pe[kQPer];      // MODE 0: the two parents' corrections
    uint32_t pp[kQPer];    // MODE 0: the two parents' codes
    auto fetch = [&](uint32_t tt) {
        int tx, ty, tz, i, j, k;
        mg_tile_xyz(L.tiles[tt], L.D, tx, ty, tz);
#pragma unroll
        for (int m = 0; m < kQPer; ++m) {
            const uint32_t sl = mg_quad_slot(map[m], tx, ty, tz, L.D, i, j, k);
            pc[m] = 0u;
            pp[m] = 0u;
            pr[m] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            pu[m] = pr[m];
            pe[m] = make_float2(0.0f, 0.0f);
            if (sl != 0xFFFFFFFFu) {
                pc[m] = *reinterpret_cast<const uint32_t*>(L.cell + sl);
                pr[m] = *reinterpret_cast<const float4*>(L.r + sl);
                if (MODE == 0) {
                    pu[m] = *reinterpret_cast<const float4*>(L.t + sl);
                    // parents of x, x+1 and of x+2, x+3: consecutive coarse cells
                    const uint32_t ps = mg_slot(i >> 1, j >> 1, k >> 1, C.D);
                    pe[m] = *reinterpret_cast<const float2*>(C.z + ps);
                    pp[m] = *reinterpret_cast<const uint16_t*>(C.cell + ps);
                } else if (MODE == 1 || MODE == 3) {
                    pu[m] = *reinterpret_cast<const float4*>(zn + sl);
                }
            }
        }
    };
    __syncthreads();  // the 1/d table
    for (uint32_t tt = blockIdx.x; tt < n; tt += gridDim.x) {
        const uint32_t key = L.tiles[tt];
        fetch(tt);
#pragma unroll
        for (int m = 0; m < kQPer; ++m) {
            const int q = tid + m * kMgThreads;
            if (q < kBoxQ) {
                const uint32_t c4 = pc[m];
                float4 r, u;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const uint32_t c = (c4 >> (8 * e)) & 0xFFu;
                    const bool fl = (c & kCellFluid) != 0;
                    const float rv = fl ? f4(pr[m], e) : 0.0f;
                    float uv = 0.0f;
                    if (fl) {
                        if (MODE == 0) {
                            // a parent that is not fluid may sit in a tile off
                            // the coarse list (stale z): it contributes nothing
                            const uint32_t cp = (pp[m] >> (8 * (e >> 1))) & 0xFFu;
                            uv = f4(pu[m], e) + ((cp & kCellFluid) ? (e < 2 ? pe[m].x : pe[m].y) : 0.0f);
                        } else if (MODE == 1) {
                            uv = f4(pu[m], e) + inv[c & 7u] * rv;
                        } else if (MODE == 3) {
                            uv = f4(pu[m], e);
                        } else {
                            uv = kMgOmega * inv[c & 7u] * rv;
                        }
                    }
                    f4set(r, e, rv);
                    f4set(u, e, uv);
                }
                cb[q] = c4;
                *reinterpret_cast<float4*>(rb + 4 * q) = r;
                *reinterpret_cast<float4*>(ub + 4 * q) = u;
            }
        }
        __syncthreads();
        for (int w = tid; w < kSw1Q; w += kMgThreads) {
            const int qd = w & 3, row = w >> 2;
            const int by = row % 10 + 1, bz = row / 10 + 1;
            const int b = 4 * qd + kBX * (by + kBY * bz);
            const float4 uc = *reinterpret_cast<const float4*>(ub + b);
            const float4 o = mg_quad_sweep(cb[b >> 2], uc, *reinterpret_cast<const float4*>(rb + b),
                                           mg_quad_nb_row<kBX, kBX * kBY>(ub, b, qd, uc), inv);
            *reinterpret_cast<float4*>(tb + 4 * qd + kBX * (row % 10 + 10 * (row / 10))) = o;
        }
        __syncthreads();
        if (tid < 128) {
            const int half = tid & 1, row = tid >> 1, ly = row & 7, lz = row >> 3;
            const int qd = 1 + half;
            const int b = 4 * qd + kBX * ((ly + 2) + kBY * (lz + 2));
            const int t = 4 * qd + kBX * ((ly + 1) + 10 * (lz + 1));
            const uint32_t zs = (key << 9) | (uint32_t)(4 * half + 8 * ly + 64 * lz);
            float4 q4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (DOT) q4 = *reinterpret_cast<const float4*>(dot.q + zs);
            const uint32_t c4 = cb[b >> 2];
            const float4 r4 = *reinterpret_cast<const float4*>(rb + b);
            const float4 tv = *reinterpret_cast<const float4*>(tb + t);
            const float4 z = mg_quad_sweep(c4, tv, r4, mg_quad_nb_pair<kBX, kBX * 10>(tb, t, half, tv), inv);
            *reinterpret_cast<float4*>(L.z + zs) = z;
            if (DOT) {
                double rz = 0.0, zq = 0.0;
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    if (!((c4 >> (8 * m)) & kCellFluid)) continue;
                    rz += (double)f4(r4, m) * (double)f4(z, m);
                    zq += (double)f4(z, m) * (double)f4(q4, m);
                }
                acc[2 * tid] += rz;
                acc[2 * tid + 1] += zq;
            }
        }
        __syncthreads();
    }
    if (DOT) {
        double out[2];
        const bool last = mg_last_cta_sum2(tid < 128 ? acc[2 * tid] : 0.0, tid < 128 ? acc[2 * tid + 1] : 0.0,
                                           dot.partials, &dot.st->ticket, out);
        if (last && tid == 0) {
            PcgState* st = dot.st;
            st->beta = dot.init ? 0.0 : (st->pq > 0.0 ? -out[1] / st->pq : 0.0);
            st->rz = out[0];
            st->rz_prev = out[0];
            st->zq = out[1];
            if (out[0] == 0.0 || !isfinite(out[0]) || !isfinite(out[1])) { st->done = 3; st->halt = 1; }
        }
    }
}

// 1 / rms(r) over the fluid cells of a level (one CTA)
__global__ void __launch_bounds__(1024) mg_scale_kernel(MgLevel L, float* inv_s, const int* halt) {
    pdl_wait();
    if (mg_halted(halt)) return;
    __shared__ double sh[32];
    const uint32_t n = *L.d_ntiles;
    double rr = 0.0, nf = 0.0;
    for (uint32_t v = threadIdx.x; v < n * 512u; v += 1024u) {
        const uint32_t s = (L.tiles[v >> 9] << 9) | (v & 511u);
        if (L.cell[s] & kCellFluid) {
            const double r = L.r[s];
            rr += r * r;
            nf += 1.0;
        }
    }
    rr = block_sum_f64<1024>(rr, sh);
    __syncthreads();
    nf = block_sum_f64<1024>(nf, sh);
    if (threadIdx.x == 0) *inv_s = rr > 0.0 ? (float)(1.0 / sqrt(rr / fmax(nf, 1.0))) : 1.0f;
}

// Jacobi-PCG on one level in one CTA (the coarsest level: at most 4096
// slots): x = A^-1 b to |r| <= tol |b| or max_iter iterations, FP32 vectors
// and FP64 dots.  r, p, q are scratch vectors of the level's size.  Used for
// the training targets of the coarsest solve.
__global__ void __launch_bounds__(1024) mg_cg_kernel(MgLevel L, const float* __restrict__ b, float* __restrict__ x,
                                                     float* __restrict__ r, float* __restrict__ p, float* __restrict__ q,
                                                     double tol, int max_iter, int* iters, const int* halt) {
    if (mg_halted(halt)) return;
    __shared__ double sh[32];
    __shared__ double bc;
    const uint32_t n = *L.d_ntiles * 512u;
    auto slot = [&](uint32_t v) { return (L.tiles[v >> 9] << 9) | (v & 511u); };
    auto bsum = [&](double v) {
        v = block_sum_f64<1024>(v, sh);
        if (threadIdx.x == 0) bc = v;
        __syncthreads();
        return bc;
    };
    double bb = 0.0, rz = 0.0;
    for (uint32_t v = threadIdx.x; v < n; v += 1024u) {
        const uint32_t s = slot(v);
        const uint8_t c = L.cell[s];
        const float bv = (c & kCellFluid) ? b[s] : 0.0f;
        x[s] = 0.0f;
        r[s] = bv;
        const float z = mg_dinv(c) * bv;
        p[s] = z;
        bb += (double)bv * bv;
        rz += (double)bv * z;
    }
    bb = bsum(bb);
    rz = bsum(rz);
    int it = 0;
    if (bb > 0.0) {
        for (it = 1; it <= max_iter; ++it) {
            double pq = 0.0;
            for (uint32_t v = threadIdx.x; v < n; v += 1024u) {
                const uint32_t s = slot(v);
                const uint8_t c = L.cell[s];
                float qv = 0.0f;
                if (c & kCellFluid) {
                    int i, j, k;
                    mg_cell_of(s >> 9, (int)(s & 511u), L.D, i, j, k);
                    const float nb = mg_nb_sum(i, j, k, L.D, L.cell, [&](uint32_t u) { return p[u]; });
                    qv = (float)(c & 7u) * p[s] - nb;
                }
                q[s] = qv;
                pq += (double)p[s] * qv;
            }
            pq = bsum(pq);
            if (!(pq > 0.0)) break;
            const float alpha = (float)(rz / pq);
            double rr = 0.0, rzn = 0.0;
            for (uint32_t v = threadIdx.x; v < n; v += 1024u) {
                const uint32_t s = slot(v);
                x[s] += alpha * p[s];
                const float rv = r[s] - alpha * q[s];
                r[s] = rv;
                rr += (double)rv * rv;
                rzn += (double)rv * (mg_dinv(L.cell[s]) * rv);
            }
            rr = bsum(rr);
            rzn = bsum(rzn);
            if (rr <= tol * tol * bb) break;
            const float beta = (float)(rzn / rz);
            rz = rzn;
            for (uint32_t v = threadIdx.x; v < n; v += 1024u) {
                const uint32_t s = slot(v);
                p[s] = mg_dinv(L.cell[s]) * r[s] + beta * p[s];
            }
            __syncthreads();
        }
    }
    if (threadIdx.x == 0 && iters) *iters = it;
}

// ------------------------------------------------------------ host side
int mg_plan(int nx, int ny, int nz, float h, MgLevel* L, int max_levels) {
    int ex = nx, ey = ny, ez = nz, levels = 0;
    float hl = h;
    while (levels < max_levels) {
        MgLevel& l = L[levels];
        l = MgLevel{};
        l.ex = ex; l.ey = ey; l.ez = ez;
        l.D.nx = (ex + 7) & ~7; l.D.ny = (ey + 7) & ~7; l.D.nz = (ez + 7) & ~7;
        l.D.tx = l.D.nx / 8; l.D.ty = l.D.ny / 8; l.D.tz = l.D.nz / 8;
        l.D.ox = l.D.oy = l.D.oz = 0.0f;
        l.D.h = hl;
        l.D.inv_h = 1.0f / hl;
        l.ntiles = (uint32_t)(l.D.tx * l.D.ty * l.D.tz);
        ++levels;
        if (ex <= kMgCoarsest && ey <= kMgCoarsest && ez <= kMgCoarsest) break;
        ex = (ex + 1) / 2; ey = (ey + 1) / 2; ez = (ez + 1) / 2;
        hl *= 2.0f;
    }
    return levels;
}

// CTAs of the smoothing kernels: five per SM (grid0 on level 0) and no more
// than the level has tiles
static int mg_grid(const MgLevel& L, int grid0, int level) {
    if (level == 0) return grid0;
    return (int)(L.ntiles < 740u ? L.ntiles : 740u);
}

int mg_build(const MgHierarchy& H, const int* halt, cudaStream_t s) {
    for (int l = 1; l < H.levels; ++l) {
        const MgLevel& C = H.L[l];
        const int g = (int)(C.ntiles < 1184u ? C.ntiles : 1184u);
        mg_coarsen_kernel<<<g, 512, 0, s>>>(H.L[l - 1], C, halt);
        mg_codes_kernel<<<g, 512, 0, s>>>(C, halt);
        // the smoothing of an intermediate level walks its tiles with fluid
        // cells (flags in C.active); the coarsest keeps every tile
        if (l + 1 < H.levels) {
            const int rc = nat_launch_fluid_tiles(C.type, C.active, C.ntiles, const_cast<uint32_t*>(C.tiles),
                                                  const_cast<uint32_t*>(C.d_ntiles), (uint64_t)C.ntiles * 512u, s);
            if (rc != FLIP_OK) return rc;
        }
    }
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int mg_down(const MgHierarchy& H, const int* halt, int grid0, cudaStream_t s, bool scale) {
    if (scale && H.levels < 2) return FLIP_ERR_ARG;
    const MgScale ns{};
    for (int l = 0; l + 1 < H.levels; ++l) {
        const int g = mg_grid(H.L[l], grid0, l);
        if (scale && l + 2 == H.levels) {
            if (2 * g > kMgScalePartials) return FLIP_ERR_ARG;
            const MgScale sc{H.scale_partials, H.scale_ticket, H.inv_s};
            FLIP_CUDA_TRY(pdl_launch(mg_down_kernel<true>, g, kMgThreads, 0, s, H.L[l], H.L[l + 1], halt, sc));
        } else {
            FLIP_CUDA_TRY(pdl_launch(mg_down_kernel<false>, g, kMgThreads, 0, s, H.L[l], H.L[l + 1], halt, ns));
        }
    }
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int mg_coarsest(const MgHierarchy& H, const float* zn, const int* halt, cudaStream_t s, bool solved) {
    const int c = H.levels - 1;
    const MgLevel& L = H.L[c];
    const int g = mg_grid(L, 740, c);
    const float* z0 = zn;
    const MgDot nd{};
    if (zn && solved) FLIP_CUDA_TRY(pdl_launch(mg_sweeps_kernel<3>, g, kMgThreads, 0, s, L, L, z0, halt, nd));
    else if (zn) FLIP_CUDA_TRY(pdl_launch(mg_sweeps_kernel<1>, g, kMgThreads, 0, s, L, L, z0, halt, nd));
    else FLIP_CUDA_TRY(pdl_launch(mg_sweeps_kernel<2>, g, kMgThreads, 0, s, L, L, z0, halt, nd));
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int mg_up(const MgHierarchy& H, const int* halt, int grid0, cudaStream_t s, const MgDot* dot) {
    if (dot && (H.levels < 2 || 2 * grid0 > 4 * kPcgBlocks)) return FLIP_ERR_ARG;  // partials: 4 x kPcgBlocks
    const MgDot nd{};
    for (int l = H.levels - 2; l >= 0; --l) {
        const int g = mg_grid(H.L[l], grid0, l);
        if (l == 0 && dot)
            FLIP_CUDA_TRY(pdl_launch(mg_sweeps_kernel<0, true>, g, kMgThreads, 0, s, H.L[l], H.L[l + 1],
                                     (const float*)nullptr, halt, *dot));
        else
            FLIP_CUDA_TRY(pdl_launch(mg_sweeps_kernel<0>, g, kMgThreads, 0, s, H.L[l], H.L[l + 1], (const float*)nullptr,
                                     halt, nd));
    }
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int mg_cg(const MgLevel& L, const float* b, float* x, float* r, float* p, float* q, double tol, int max_iter, int* iters,
          cudaStream_t s, const int* halt) {
    mg_cg_kernel<<<1, 1024, 0, s>>>(L, b, x, r, p, q, tol, max_iter, iters, halt);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int mg_input_scale(const MgHierarchy& H, const int* halt, cudaStream_t s) {
    FLIP_CUDA_TRY(pdl_launch(mg_scale_kernel, 1, 1024, 0, s, H.L[H.levels - 1], H.inv_s, halt));
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

}  // namespace flip
