// mg.cu -- V-cycle kernels of the multilevel learned preconditioner (mg.cuh).
//
// Every level is tile-blocked like the solver's grid (slot = tile * 512 +
// (i & 7) + 8 (j & 7) + 64 (k & 7)).  The smoothing kernels walk a tile list
// with one CTA of 512 threads per tile and one thread per cell; neighbours
// come from global memory (the coarse levels are small enough to stay in L2).
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
// 12^3 box of its tile and a 2-cell halo in shared memory (cell codes, r and
// the vector the sweeps start from); the first sweep is evaluated on the
// 10^3 box of the tile and a 1-cell halo, the second (or the residual) on
// the tile.  A neighbour that is not fluid contributes nothing, so halo cells
// outside the grid or in tiles off the level's list (code 0) need no test
// beyond the code.
constexpr int kB12 = 12 * 12 * 12;
constexpr int kB10 = 10 * 10 * 10;
__device__ __forceinline__ void mg_origin(uint32_t key, const NatDims& D, int& ox, int& oy, int& oz) {
    const uint32_t tyz = key / (uint32_t)D.tx;
    ox = 8 * (int)(key - tyz * (uint32_t)D.tx);
    oy = 8 * (int)(tyz % (uint32_t)D.ty);
    oz = 8 * (int)(tyz / (uint32_t)D.ty);
}
// sum of the fluid neighbours' values of box cell b (row strides sx, sy, sz
// = 1, W, W*W of a W-wide box), codes from the 12^3 box at b12
__device__ __forceinline__ float mg_box_nb(const uint8_t* cb, int b12, const float* vb, int b, int W) {
    const int W2 = W * W;
    float s = 0.0f;
    if (cb[b12 - 1] & kCellFluid) s += vb[b - 1];
    if (cb[b12 + 1] & kCellFluid) s += vb[b + 1];
    if (cb[b12 - 12] & kCellFluid) s += vb[b - W];
    if (cb[b12 + 12] & kCellFluid) s += vb[b + W];
    if (cb[b12 - 144] & kCellFluid) s += vb[b - W2];
    if (cb[b12 + 144] & kCellFluid) s += vb[b + W2];
    return s;
}
__device__ __forceinline__ int b12_of10(int v) {  // 10^3 box index -> 12^3 box index
    const int x = v % 10, y = (v / 10) % 10, z = v / 100;
    return (x + 1) + 12 * ((y + 1) + 12 * (z + 1));
}

// Both kernels run 256 threads per CTA (four CTAs per SM) and keep the
// next tile's box loads in flight while the current tile computes.  A thread
// owns up to seven box cells; which neighbour tile (3 x 3 x 3 around the
// tile) and which slot in it each one is does not depend on the tile and is
// worked out once.  Codes and values are loaded without waiting for the code
// (every slot inside the grid is a valid address) and masked to the fluid
// cells when they go to shared memory, where every vector is then zero off
// the fluid cells: a neighbour sum needs no test.  1/d comes from a shared
// table.
constexpr int kMgThreads = 256;
constexpr int kBoxPer = (kB12 + kMgThreads - 1) / kMgThreads;  // 7
constexpr int kB10Per = (kB10 + kMgThreads - 1) / kMgThreads;  // 4

// box cell v -> (neighbour tile offset + 1 per axis, local slot), packed
// as local | (qx + 1) << 9 | (qy + 1) << 11 | (qz + 1) << 13; -1 past the box
__device__ __forceinline__ int mg_box_map(int v) {
    if (v >= kB12) return -1;
    const int x = v % 12 - 2, y = (v / 12) % 12 - 2, z = v / 144 - 2;
    const int qx = (x + 8) / 8 - 1, qy = (y + 8) / 8 - 1, qz = (z + 8) / 8 - 1;
    const int local = (x - 8 * qx) | ((y - 8 * qy) << 3) | ((z - 8 * qz) << 6);
    return local | ((qx + 1) << 9) | ((qy + 1) << 11) | ((qz + 1) << 13);
}
// slot of a mapped box cell around the tile at tile coordinates (tx, ty, tz),
// or UINT32_MAX outside the grid; (i, j, k) of the cell out
__device__ __forceinline__ uint32_t mg_map_slot(int map, int tx, int ty, int tz, const NatDims& D, int& i, int& j, int& k) {
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
__device__ __forceinline__ float mg_sum6(const float* vb, int b, int W) {
    return ((vb[b - 1] + vb[b + 1]) + (vb[b - W] + vb[b + W])) + (vb[b - W * W] + vb[b + W * W]);
}
__device__ __forceinline__ void mg_inv_table(float* inv) {
    if (threadIdx.x < 8) {
        const float d = (float)threadIdx.x;
        inv[threadIdx.x] = threadIdx.x ? 1.0f / d : 0.0f;
    }
}

// pre-smoothing and restriction of level F into C:
//   t1 = w D^-1 r, t = t1 + w D^-1 (r - A t1) (kept in F.t),
//   C.r[parent] = 1/2 sum over the 8 children of r - A t (fluid parents; the
//   parents of a tile are all written by it, and parents of tiles off the
//   list are never fluid)
__global__ void __launch_bounds__(kMgThreads, 4) mg_down_kernel(MgLevel F, MgLevel C, const int* halt) {
    if (mg_halted(halt)) return;
    __shared__ uint8_t cb[kB12];
    __shared__ float rb[kB12];
    __shared__ float t1b[kB12];
    __shared__ float tb[kB10];
    __shared__ float S[512];
    __shared__ float inv[8];
    mg_inv_table(inv);
    const int tid = threadIdx.x;
    int map[kBoxPer], b10m[kB10Per];
#pragma unroll
    for (int m = 0; m < kBoxPer; ++m) map[m] = mg_box_map(tid + m * kMgThreads);
#pragma unroll
    for (int m = 0; m < kB10Per; ++m) b10m[m] = tid + m * kMgThreads < kB10 ? b12_of10(tid + m * kMgThreads) : -1;
    const uint32_t n = *F.d_ntiles;
    uint8_t pc[kBoxPer];
    float pr[kBoxPer];
    auto fetch = [&](uint32_t tt) {
        int tx, ty, tz, i, j, k;
        mg_tile_xyz(F.tiles[tt], F.D, tx, ty, tz);
#pragma unroll
        for (int m = 0; m < kBoxPer; ++m) {
            const uint32_t sl = mg_map_slot(map[m], tx, ty, tz, F.D, i, j, k);
            pc[m] = 0;
            pr[m] = 0.0f;
            if (sl != 0xFFFFFFFFu) {
                pc[m] = F.cell[sl];
                pr[m] = F.r[sl];
            }
        }
    };
    uint32_t tt = blockIdx.x;
    if (tt < n) fetch(tt);
    __syncthreads();  // the 1/d table
    for (; tt < n; tt += gridDim.x) {
        const uint32_t key = F.tiles[tt];
#pragma unroll
        for (int m = 0; m < kBoxPer; ++m) {
            const int v = tid + m * kMgThreads;
            if (v < kB12) {
                const uint8_t c = pc[m];
                const bool fl = (c & kCellFluid) != 0;
                const float r = fl ? pr[m] : 0.0f;
                cb[v] = c;
                rb[v] = r;
                t1b[v] = kMgOmega * inv[c & 7u] * r;
            }
        }
        __syncthreads();
        if (tt + gridDim.x < n) fetch(tt + gridDim.x);  // in flight during this tile's work
#pragma unroll
        for (int m = 0; m < kB10Per; ++m) {
            const int b = b10m[m];
            if (b < 0) continue;
            const uint8_t c = cb[b];
            const float t1 = t1b[b];
            tb[tid + m * kMgThreads] = (c & kCellFluid) ? t1 + kMgOmega * inv[c & 7u] * (rb[b] - ((float)(c & 7u) * t1 - mg_sum6(t1b, b, 12))) : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int cidx = tid + h * kMgThreads;
            const int li = cidx & 7, lj = (cidx >> 3) & 7, lk = cidx >> 6;
            const int b12 = (li + 2) + 12 * ((lj + 2) + 12 * (lk + 2));
            const int b10 = (li + 1) + 10 * ((lj + 1) + 10 * (lk + 1));
            const uint8_t c = cb[b12];
            const float tv = tb[b10];
            F.t[(key << 9) | cidx] = tv;
            S[cidx] = (c & kCellFluid) ? rb[b12] - ((float)(c & 7u) * tv - mg_sum6(tb, b10, 10)) : 0.0f;
        }
        __syncthreads();
        if (tid < 64) {  // the (even, even, even) child of each 2^3 block
            int tx, ty, tz;
            mg_tile_xyz(key, F.D, tx, ty, tz);
            const int pi = tid & 3, pj = (tid >> 2) & 3, pk = tid >> 4;
            const int b = 2 * pi + 16 * pj + 128 * pk;
            const float sum = ((S[b] + S[b + 1]) + (S[b + 8] + S[b + 9])) + ((S[b + 64] + S[b + 65]) + (S[b + 72] + S[b + 73]));
            const uint32_t p = mg_slot(4 * tx + pi, 4 * ty + pj, 4 * tz + pk, C.D);
            C.r[p] = (C.cell[p] & kCellFluid) ? 0.5f * sum : 0.0f;
        }
        __syncthreads();
    }
}

// two damped Jacobi sweeps from a start vector u: t2 = u + w D^-1 (r - A u),
// L.z = t2 + w D^-1 (r - A t2).  MODE 0: u = L.t + C.z[parent] (prolongation
// of the coarse correction; post-smoothing); MODE 1: u = zn + D^-1 r (the
// coarsest level with the network output zn); MODE 2: u = w D^-1 r (the
// coarsest level without the network).
template <int MODE>
__global__ void __launch_bounds__(kMgThreads, 4) mg_sweeps_kernel(MgLevel L, MgLevel C, const float* __restrict__ zn,
                                                                  const int* halt) {
    if (mg_halted(halt)) return;
    __shared__ uint8_t cb[kB12];
    __shared__ float rb[kB12];
    __shared__ float ub[kB12];
    __shared__ float tb[kB10];
    __shared__ float inv[8];
    mg_inv_table(inv);
    const int tid = threadIdx.x;
    int map[kBoxPer], b10m[kB10Per];
#pragma unroll
    for (int m = 0; m < kBoxPer; ++m) map[m] = mg_box_map(tid + m * kMgThreads);
#pragma unroll
    for (int m = 0; m < kB10Per; ++m) b10m[m] = tid + m * kMgThreads < kB10 ? b12_of10(tid + m * kMgThreads) : -1;
    const uint32_t n = *L.d_ntiles;
    uint8_t pc[kBoxPer];
    float pr[kBoxPer], pu[kBoxPer];
    auto fetch = [&](uint32_t tt) {
        int tx, ty, tz, i, j, k;
        mg_tile_xyz(L.tiles[tt], L.D, tx, ty, tz);
#pragma unroll
        for (int m = 0; m < kBoxPer; ++m) {
            const uint32_t sl = mg_map_slot(map[m], tx, ty, tz, L.D, i, j, k);
            pc[m] = 0;
            pr[m] = 0.0f;
            pu[m] = 0.0f;
            if (sl != 0xFFFFFFFFu) {
                pc[m] = L.cell[sl];
                pr[m] = L.r[sl];
                if (MODE == 0) {
                    // the parent's correction; a parent that is not fluid
                    // may sit in a tile off the coarse list (stale z)
                    const uint32_t ps = mg_slot(i >> 1, j >> 1, k >> 1, C.D);
                    pu[m] = L.t[sl] + ((C.cell[ps] & kCellFluid) ? C.z[ps] : 0.0f);
                }
                else if (MODE == 1) pu[m] = zn[sl];
            }
        }
    };
    uint32_t tt = blockIdx.x;
    if (tt < n) fetch(tt);
    __syncthreads();  // the 1/d table
    for (; tt < n; tt += gridDim.x) {
        const uint32_t key = L.tiles[tt];
#pragma unroll
        for (int m = 0; m < kBoxPer; ++m) {
            const int v = tid + m * kMgThreads;
            if (v < kB12) {
                const uint8_t c = pc[m];
                const bool fl = (c & kCellFluid) != 0;
                const float r = fl ? pr[m] : 0.0f;
                float u = 0.0f;
                if (fl) u = MODE == 0 ? pu[m] : (MODE == 1 ? pu[m] + inv[c & 7u] * r : kMgOmega * inv[c & 7u] * r);
                cb[v] = c;
                rb[v] = r;
                ub[v] = u;
            }
        }
        __syncthreads();
        if (tt + gridDim.x < n) fetch(tt + gridDim.x);  // in flight during this tile's work
#pragma unroll
        for (int m = 0; m < kB10Per; ++m) {
            const int b = b10m[m];
            if (b < 0) continue;
            const uint8_t c = cb[b];
            const float u = ub[b];
            tb[tid + m * kMgThreads] = (c & kCellFluid) ? u + kMgOmega * inv[c & 7u] * (rb[b] - ((float)(c & 7u) * u - mg_sum6(ub, b, 12))) : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int cidx = tid + h * kMgThreads;
            const int li = cidx & 7, lj = (cidx >> 3) & 7, lk = cidx >> 6;
            const int b12 = (li + 2) + 12 * ((lj + 2) + 12 * (lk + 2));
            const int b10 = (li + 1) + 10 * ((lj + 1) + 10 * (lk + 1));
            const uint8_t c = cb[b12];
            const float tv = tb[b10];
            L.z[(key << 9) | cidx] =
                (c & kCellFluid) ? tv + kMgOmega * inv[c & 7u] * (rb[b12] - ((float)(c & 7u) * tv - mg_sum6(tb, b10, 10))) : 0.0f;
        }
        __syncthreads();
    }
}

// 1 / rms(r) over the fluid cells of a level (one CTA)
__global__ void __launch_bounds__(1024) mg_scale_kernel(MgLevel L, float* inv_s, const int* halt) {
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
                                                     double tol, int max_iter, int* iters) {
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
        l.ntiles = (uint32_t)(l.D.tx * l.D.ty * l.D.tz);
        ++levels;
        if (ex <= kMgCoarsest && ey <= kMgCoarsest && ez <= kMgCoarsest) break;
        ex = (ex + 1) / 2; ey = (ey + 1) / 2; ez = (ez + 1) / 2;
        hl *= 2.0f;
    }
    return levels;
}

// CTAs of the smoothing kernels: four per SM (grid0 on level 0) and no more
// than the level has tiles
static int mg_grid(const MgLevel& L, int grid0, int level) {
    if (level == 0) return grid0;
    return (int)(L.ntiles < 592u ? L.ntiles : 592u);
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

int mg_down(const MgHierarchy& H, const int* halt, int grid0, cudaStream_t s) {
    for (int l = 0; l + 1 < H.levels; ++l)
        mg_down_kernel<<<mg_grid(H.L[l], grid0, l), kMgThreads, 0, s>>>(H.L[l], H.L[l + 1], halt);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int mg_coarsest(const MgHierarchy& H, const float* zn, const int* halt, cudaStream_t s) {
    const int c = H.levels - 1;
    const MgLevel& L = H.L[c];
    const int g = mg_grid(L, 592, c);
    if (zn) mg_sweeps_kernel<1><<<g, kMgThreads, 0, s>>>(L, L, zn, halt);
    else mg_sweeps_kernel<2><<<g, kMgThreads, 0, s>>>(L, L, nullptr, halt);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int mg_up(const MgHierarchy& H, const int* halt, int grid0, cudaStream_t s) {
    for (int l = H.levels - 2; l >= 0; --l)
        mg_sweeps_kernel<0><<<mg_grid(H.L[l], grid0, l), kMgThreads, 0, s>>>(H.L[l], H.L[l + 1], nullptr, halt);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int mg_cg(const MgLevel& L, const float* b, float* x, float* r, float* p, float* q, double tol, int max_iter, int* iters,
          cudaStream_t s) {
    mg_cg_kernel<<<1, 1024, 0, s>>>(L, b, x, r, p, q, tol, max_iter, iters);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int mg_input_scale(const MgHierarchy& H, const int* halt, cudaStream_t s) {
    mg_scale_kernel<<<1, 1024, 0, s>>>(H.L[H.levels - 1], H.inv_s, halt);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

}  // namespace flip
