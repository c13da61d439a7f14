// native.cu -- the native-mode fluid step on sm_100a (FP32 state).
//
// Grid layout.  Voxel grids are dense, allocated once for the whole box
// (256^3 voxels are 64 MiB per float field; a B200 holds 180 GB) and stored
// tile-blocked: slot = tile*512 + (i&7) + 8*(j&7) + 64*(k&7), tile =
// (i>>3) + TX*((j>>3) + TY*(k>>3)).  A tile's 512 values are one contiguous
// 2 KiB block, neighbours are address arithmetic (no index tables), and only
// the tiles that hold particles (or touch their stencils) are visited.  Face
// (i,j,k) of a velocity component is the negative face of cell (i,j,k); the
// positive box walls are implicit zeros.
//
// Particles are SoA float arrays sorted by tile every step (sort.cu), so a
// CTA working on one tile reads one contiguous particle range.
#include <cudaTypedefs.h>
#include <mutex>
#include "common.cuh"
#include "native.cuh"
#include "tma.cuh"

namespace flip {

__device__ __forceinline__ uint32_t nslot(int i, int j, int k, const NatDims& D) {
    uint32_t t = (uint32_t)((i >> 3) + D.tx * ((j >> 3) + D.ty * (k >> 3)));
    return (t << 9) | (uint32_t)((i & 7) | ((j & 7) << 3) | ((k & 7) << 6));
}
// cell of grid coordinate g = (p - o) / h, clamped into [0, n)
__device__ __forceinline__ int nat_cell_g(float g, int n) {
    float t = floorf(g);
    int c = (t >= (float)n) ? n - 1 : (int)t;
    if (!(t > 0.0f)) c = 0;
    return c;
}
// grid coordinate of a position on one axis; the one form every kernel uses
// for cells, keys and stencils, so that they agree on which cell holds a
// particle (exact, like a division, when h is a power of two)
__device__ __forceinline__ float nat_grid_coord(float p, float o, float inv_h) { return __fmul_rn(__fsub_rn(p, o), inv_h); }
__device__ __forceinline__ int nat_cell(float p, float o, float inv_h, int n) { return nat_cell_g(nat_grid_coord(p, o, inv_h), n); }
__device__ __forceinline__ uint8_t nat_type(const uint8_t* type, int i, int j, int k, const NatDims& D) {
    if (i < 0 || j < 0 || k < 0 || i >= D.nx || j >= D.ny || k >= D.nz) return kSolid;
    return type[nslot(i, j, k, D)];
}
// stencil base and weight on one axis of M + 1 nodes: s clamped into
// [0, M], base floor(s) capped at M - 1 (computed as a float, which is exact
// for these small integers), weight s - base
__device__ __forceinline__ void nat_axis(float s, int M, int& i0, float& f) {
    s = fminf(fmaxf(s, 0.0f), (float)M);
    const float b = fminf(floorf(s), (float)(M - 1));
    i0 = (int)b;
    f = s - b;
}
// trilinear stencil of component c at grid coordinates (gx, gy, gz)
__device__ __forceinline__ void nat_stencil(int c, float gx, float gy, float gz, const NatDims& D, int& i0, int& j0, int& k0,
                                            float& fx, float& fy, float& fz) {
    nat_axis(c == 0 ? gx : gx - 0.5f, c == 0 ? D.nx : D.nx - 1, i0, fx);
    nat_axis(c == 1 ? gy : gy - 0.5f, c == 1 ? D.ny : D.ny - 1, j0, fy);
    nat_axis(c == 2 ? gz : gz - 0.5f, c == 2 ? D.nz : D.nz - 1, k0, fz);
}
__device__ __forceinline__ bool nat_wall(int c, int i, int j, int k, const NatDims& D) {
    if (c == 0) return i == 0 || i == D.nx;
    if (c == 1) return j == 0 || j == D.ny;
    return k == 0 || k == D.nz;
}

// ------------------------------------------------------------- binning
__global__ void nat_keys_kernel(const float* __restrict__ px, const float* __restrict__ py, const float* __restrict__ pz,
                                uint64_t n, NatDims D, uint32_t* __restrict__ keys) {
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int i = nat_cell(px[p], D.ox, D.inv_h, D.nx), j = nat_cell(py[p], D.oy, D.inv_h, D.ny), k = nat_cell(pz[p], D.oz, D.inv_h, D.nz);
    keys[p] = (uint32_t)((i >> 3) + D.tx * ((j >> 3) + D.ty * (k >> 3)));
}

// gather of the six state arrays through the sort permutation
__global__ void nat_gather_kernel(const uint32_t* __restrict__ perm, uint64_t n, const float* __restrict__ a0,
                                  const float* __restrict__ a1, const float* __restrict__ a2, const float* __restrict__ a3,
                                  const float* __restrict__ a4, const float* __restrict__ a5, float* __restrict__ b0,
                                  float* __restrict__ b1, float* __restrict__ b2, float* __restrict__ b3,
                                  float* __restrict__ b4, float* __restrict__ b5) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t s = perm[i];
    if (s >= n) s = (uint32_t)i;  // a valid permutation always has s < n
    b0[i] = __ldg(a0 + s); b1[i] = __ldg(a1 + s); b2[i] = __ldg(a2 + s);
    b3[i] = __ldg(a3 + s); b4[i] = __ldg(a4 + s); b5[i] = __ldg(a5 + s);
}

// ------------------------------------------------------------------ P2G
// One CTA per occupied tile (persistent loop) accumulates the trilinear
// weights (and weighted velocities) of the tile's particles into a
// shared-memory box of 10^3 nodes per component -- the tile plus the
// one-node halo its stencils reach -- and adds the box to the global grids;
// it also marks the cells that hold particles.
//
// A thread owns one cell of the tile.  The tile's particles are first sorted
// by cell inside the CTA (a counting sort in shared memory: one integer
// atomic per particle), with their grid coordinates kept in shared memory in
// the sorted order.  Then each thread walks its cell's particles and keeps,
// per velocity component, the 2 x 3 x 3 node sums that any particle of that
// cell can reach in registers (36 floats: two nodes along the component's own
// axis, three along each staggered axis, where the stencil's base is the cell
// or the one below).  The sums go into the box in 18 phases, one node offset
// per phase, so that within a phase no two threads touch one node: plain
// shared-memory adds, no atomics.  FP32 sums, as the oracle's comparison
// assumes (relative precision even for the tiny weights of a node that only
// one far particle reaches; a fixed-point accumulator loses exactly those).
// A float-atomic scatter (a thread per particle, 48 shared atomics each) ran
// 2-2.5x slower.
constexpr int kBox = 10;
constexpr int kBoxN = kBox * kBox * kBox;
constexpr int kPcThreads = 512;         // one thread per cell of the tile
constexpr int kPcChunk = 4096;          // particles sorted per round (a denser tile takes several)
constexpr int kPcPer = kPcChunk / kPcThreads;
// Sorted slot j (16 bytes) lives at j + j / 8: with about eight particles a
// cell, the threads of a warp (consecutive cells) read slots about eight
// apart, and the eight threads of a quarter warp, whose 16-byte reads share
// one pass over the banks, would otherwise hit the same four banks; one slot
// of padding per eight spreads them over all 32.
constexpr int kPcSlots = kPcChunk + kPcChunk / 8;
__device__ __forceinline__ uint32_t pc_slot(uint32_t j) { return j + (j >> 3); }
struct P2GCellSmem {
    float m[3][kBoxN], w[3][kBoxN];     // the box: momentum and weight sums per component
    float4 gq[kPcSlots];                // per sorted slot: the particle's grid coordinates and
                                        // (w, as bits) its index within the round
    uint32_t cnt[kPcThreads], off[kPcThreads];
    uint32_t scan[kPcThreads / 32 + 1];
};

__global__ void __launch_bounds__(kPcThreads, 2) nat_p2g_cells_kernel(
    const uint32_t* __restrict__ tile_keys, const uint32_t* __restrict__ starts, const uint32_t* __restrict__ d_ntiles,
    uint64_t n, const float* __restrict__ px, const float* __restrict__ py, const float* __restrict__ pz,
    const float* __restrict__ vx, const float* __restrict__ vy, const float* __restrict__ vz, NatDims D,
    float* __restrict__ mu, float* __restrict__ mv, float* __restrict__ mw, float* __restrict__ wu,
    float* __restrict__ wv, float* __restrict__ ww, uint8_t* __restrict__ type) {
    extern __shared__ __align__(16) unsigned char pc_smem[];
    P2GCellSmem& S = *reinterpret_cast<P2GCellSmem*>(pc_smem);
    const int tid = threadIdx.x;
    const uint32_t ntiles = *d_ntiles;
    const float* P[3] = {px, py, pz};
    float* gm[3] = {mu, mv, mw};
    float* gw[3] = {wu, wv, ww};
    const float o[3] = {D.ox, D.oy, D.oz};
    const int nn[3] = {D.nx, D.ny, D.nz};
    const int lc[3] = {tid & 7, (tid >> 3) & 7, tid >> 6};  // this thread's cell in the tile
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        for (int l = tid; l < 3 * kBoxN; l += kPcThreads) {
            (&S.m[0][0])[l] = 0.0f;
            (&S.w[0][0])[l] = 0.0f;
        }
        const uint32_t key = tile_keys[t];
        const int tc[3] = {(int)(key % D.tx), (int)((key / D.tx) % D.ty), (int)(key / (D.tx * D.ty))};
        const int cell[3] = {8 * tc[0] + lc[0], 8 * tc[1] + lc[1], 8 * tc[2] + lc[2]};
        const uint64_t start = starts[t];
        const uint64_t end = (t + 1 < ntiles) ? starts[t + 1] : n;
        for (uint64_t r0 = start; r0 < end; r0 += kPcChunk) {
            const uint32_t m = (uint32_t)min((uint64_t)kPcChunk, end - r0);
            S.cnt[tid] = 0u;
            __syncthreads();
            // counting sort of the round's particles by cell
            uint32_t slot[kPcPer];
#pragma unroll
            for (int i = 0; i < kPcPer; ++i) {
                const uint32_t q = (uint32_t)(tid + kPcThreads * i);
                slot[i] = 0xFFFFFFFFu;
                if (q < m) {
                    const uint64_t p = r0 + q;
                    int c[3];
#pragma unroll
                    for (int a = 0; a < 3; ++a) c[a] = nat_cell(P[a][p], o[a], D.inv_h, nn[a]);
                    type[nslot(c[0], c[1], c[2], D)] = kFluid;
                    // a particle of this tile's segment lies in one of its cells
                    const int l0 = c[0] - 8 * tc[0], l1 = c[1] - 8 * tc[1], l2 = c[2] - 8 * tc[2];
                    if ((unsigned)l0 < 8u && (unsigned)l1 < 8u && (unsigned)l2 < 8u) {
                        const uint32_t cl = (uint32_t)(l0 + 8 * l1 + 64 * l2);
                        slot[i] = cl | (atomicAdd(&S.cnt[cl], 1u) << 9);
                    }
                }
            }
            __syncthreads();
            uint32_t total;
            S.off[tid] = block_exclusive_scan<kPcThreads>(S.cnt[tid], S.scan, &total);
            __syncthreads();
            // the sorted slots: particle index and grid coordinates (the same
            // form nat_cell used above), so that the three component passes
            // below read them from shared memory
#pragma unroll
            for (int i = 0; i < kPcPer; ++i)
                if (slot[i] != 0xFFFFFFFFu) {
                    const uint32_t q = (uint32_t)(tid + kPcThreads * i), at = S.off[slot[i] & 511u] + (slot[i] >> 9);
                    S.gq[pc_slot(at)] = make_float4(nat_grid_coord(P[0][r0 + q], o[0], D.inv_h),
                                                    nat_grid_coord(P[1][r0 + q], o[1], D.inv_h),
                                                    nat_grid_coord(P[2][r0 + q], o[2], D.inv_h), __uint_as_float(q));
                }
            __syncthreads();
            const uint32_t b0 = S.off[tid], b1 = b0 + S.cnt[tid];
            // the three components unrolled: every axis choice below is a constant
#pragma unroll
            for (int comp = 0; comp < 3; ++comp) {
                // the component's own axis and the two others in order (a1 < a2)
                const int no = comp == 0 ? D.nx : (comp == 1 ? D.ny : D.nz);
                const int n1 = comp == 0 ? D.ny : D.nx, n2 = comp == 2 ? D.ny : D.nz;
                const int c1 = comp == 0 ? cell[1] : cell[0], c2 = comp == 2 ? cell[1] : cell[2];
                const float* __restrict__ vc = comp == 0 ? vx : (comp == 1 ? vy : vz);
                // Every particle of the walk lies in this thread's cell, so the
                // stencil's bases are constants of the thread: along the own
                // axis the cell co (weights 1 - f, f with f = sat(g - co));
                // along a staggered axis the cell or the one below, chosen by
                // the sign of f' = g - (c + 1/2), with the weights
                // max(-f', 0), 1 - |f'|, max(f', 0) on the nodes c - 1, c,
                // c + 1.  At the first and last cell f' is clamped at 0, where
                // the stencil's clamp puts all the weight on the cell's own
                // node.  The values equal those of nat_stencil bit for bit
                // (every subtraction here is exact; 1 - |f'| rounds as 1 - f
                // does there).  The own axis's wall faces take no weight: the
                // flush below skips them.
                const int co = comp == 0 ? cell[0] : (comp == 1 ? cell[1] : cell[2]);
                const float cof = (float)co, c1h = (float)c1 + 0.5f, c2h = (float)c2 + 0.5f;
                const float lo1 = c1 == 0 ? 0.0f : -1.0f, hi1 = c1 == n1 - 1 ? 0.0f : 1.0f;
                const float lo2 = c2 == 0 ? 0.0f : -1.0f, hi2 = c2 == n2 - 1 ? 0.0f : 1.0f;
                float am[18], aw[18];
#pragma unroll
                for (int k = 0; k < 18; ++k) am[k] = aw[k] = 0.0f;
                for (uint32_t j = b0; j < b1; ++j) {
                    const float4 gq = S.gq[pc_slot(j)];
                    const uint64_t p = r0 + __float_as_uint(gq.w);
                    const float gx = gq.x, gy = gq.y, gz = gq.z;
                    const float go = comp == 0 ? gx : (comp == 1 ? gy : gz);
                    const float g1 = comp == 0 ? gy : gx, g2 = comp == 2 ? gy : gz;
                    const float v = vc[p];
                    const float fo = __saturatef(go - cof);
                    const float wo0 = 1.0f - fo, wo1 = fo;
                    const float f1 = fminf(fmaxf(g1 - c1h, lo1), hi1), f2 = fminf(fmaxf(g2 - c2h, lo2), hi2);
                    const float w1[3] = {fmaxf(-f1, 0.0f), 1.0f - fabsf(f1), fmaxf(f1, 0.0f)};
                    const float w2[3] = {fmaxf(-f2, 0.0f), 1.0f - fabsf(f2), fmaxf(f2, 0.0f)};
                    const float wv0 = wo0 * v, wv1 = wo1 * v;
#pragma unroll
                    for (int d2 = 0; d2 < 3; ++d2)
#pragma unroll
                        for (int d1 = 0; d1 < 3; ++d1) {
                            const float w12 = w1[d1] * w2[d2];
                            const int k = 2 * (d1 + 3 * d2);
                            aw[k] = fmaf(wo0, w12, aw[k]);
                            am[k] = fmaf(wv0, w12, am[k]);
                            aw[k + 1] = fmaf(wo1, w12, aw[k + 1]);
                            am[k + 1] = fmaf(wv1, w12, am[k + 1]);
                        }
                }
                // the wall faces of the own axis (face 0 below the first cell,
                // face n above the last) keep no weight
                if (co == 0) {
#pragma unroll
                    for (int k = 0; k < 18; k += 2) aw[k] = 0.0f;
                }
                if (co == no - 1) {
#pragma unroll
                    for (int k = 1; k < 18; k += 2) aw[k] = 0.0f;
                }
                // 18 phases: in phase k every thread adds its node k; at one
                // offset no two cells share a node.  Box origin: tile origin - 1.
                const int lo = lc[comp == 0 ? 0 : (comp == 1 ? 1 : 2)] + 1;
                const int l1 = comp == 0 ? lc[1] : lc[0], l2 = comp == 2 ? lc[1] : lc[2];
                float* __restrict__ bm = S.m[comp];
                float* __restrict__ bw = S.w[comp];
#pragma unroll
                for (int d2 = 0; d2 < 3; ++d2)
#pragma unroll
                    for (int d1 = 0; d1 < 3; ++d1)
#pragma unroll
                        for (int d0 = 0; d0 < 2; ++d0) {
                            const int k = d0 + 2 * (d1 + 3 * d2);
                            const int io = lo + d0, i1 = l1 + d1, i2 = l2 + d2;
                            const int l = comp == 0 ? io + kBox * (i1 + kBox * i2)
                                                    : (comp == 1 ? i1 + kBox * (io + kBox * i2) : i1 + kBox * (i2 + kBox * io));
                            if (aw[k] != 0.0f) {
                                bm[l] += am[k];
                                bw[l] += aw[k];
                            }
                            __syncthreads();
                        }
            }
        }
        // the box onto the global grids (halo nodes are shared with the
        // neighbouring tiles: atomics)
        for (int l = tid; l < kBoxN; l += kPcThreads) {
            const int li = l % kBox, lj = (l / kBox) % kBox, lk = l / (kBox * kBox);
            const int i = 8 * tc[0] - 1 + li, j = 8 * tc[1] - 1 + lj, k = 8 * tc[2] - 1 + lk;
            if (i < 0 || j < 0 || k < 0 || i >= D.nx || j >= D.ny || k >= D.nz) continue;
            const uint32_t s = nslot(i, j, k, D);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float w = S.w[c][l];
                if (w != 0.0f) {
                    atomicAdd(gw[c] + s, w);
                    atomicAdd(gm[c] + s, S.m[c][l]);
                }
            }
        }
        __syncthreads();
    }
}

// packed coordinates tx | ty << 10 | tz << 20 of each occupied tile
__global__ void nat_tile_coords_kernel(const uint32_t* __restrict__ tile_keys, const uint32_t* __restrict__ d_ntiles,
                                       NatDims D, uint32_t* __restrict__ coords) {
    const uint32_t ntiles = *d_ntiles;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x) {
        const uint32_t key = tile_keys[t];
        coords[t] = (key % D.tx) | (((key / D.tx) % D.ty) << 10) | ((key / (D.tx * D.ty)) << 20);
    }
}

// ------------------------------------------------ standalone Poisson problems
// Cell types and right-hand side of a pressure problem on the whole box:
// solid inside any sphere (cx, cy, cz, r in voxels), fluid below the surface
// height, air above; b = -div(u) on fluid cells for u = sum of Gaussian
// velocity impulses (cx, cy, cz, sigma, ax, ay, az) plus gravity*dt on the
// y faces next to fluid, with faces touching a solid cell or a wall at zero.
__device__ __forceinline__ bool gen_solid(float x, float y, float z, const float4* sph, int nsph) {
    for (int q = 0; q < nsph; ++q) {
        const float4 s = sph[q];
        const float dx = x - s.x, dy = y - s.y, dz = z - s.z;
        if (dx * dx + dy * dy + dz * dz < s.w * s.w) return true;
    }
    return false;
}
__device__ __forceinline__ uint8_t gen_type(int i, int j, int k, const NatDims& D, float surface, const float4* sph,
                                            int nsph) {
    if (i < 0 || j < 0 || k < 0 || i >= D.nx || j >= D.ny || k >= D.nz) return kSolid;
    if (gen_solid(i + 0.5f, j + 0.5f, k + 0.5f, sph, nsph)) return kSolid;
    return (j + 0.5f < surface) ? kFluid : kAir;
}
__device__ __forceinline__ float gen_face(int c, int i, int j, int k, const NatDims& D, float surface, const float4* sph,
                                          int nsph, const float* imp, int nimp, float gdt) {
    // face c of cell (i,j,k): between (i,j,k) - e_c and (i,j,k)
    const uint8_t tb = gen_type(i, j, k, D, surface, sph, nsph);
    const uint8_t ta = gen_type(i - (c == 0), j - (c == 1), k - (c == 2), D, surface, sph, nsph);
    if (ta == kSolid || tb == kSolid) return 0.0f;
    const float x = i + (c == 0 ? 0.0f : 0.5f), y = j + (c == 1 ? 0.0f : 0.5f), z = k + (c == 2 ? 0.0f : 0.5f);
    float u = 0.0f;
    for (int q = 0; q < nimp; ++q) {
        const float* m = imp + 7 * q;
        const float dx = x - m[0], dy = y - m[1], dz = z - m[2];
        u += m[4 + c] * __expf(-(dx * dx + dy * dy + dz * dz) / (2.0f * m[3] * m[3]));
    }
    if (c == 1 && (ta == kFluid || tb == kFluid)) u += gdt;
    return u;
}
__global__ void nat_poisson_gen_kernel(NatDims D, float surface, const float4* __restrict__ sph, int nsph,
                                       const float* __restrict__ imp, int nimp, float gdt, uint8_t* __restrict__ type,
                                       float* __restrict__ b, uint64_t nslots) {
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const uint32_t tile = (uint32_t)(s >> 9), l = (uint32_t)(s & 511u);
    const int i = 8 * (int)(tile % D.tx) + (int)(l & 7u), j = 8 * (int)((tile / D.tx) % D.ty) + (int)((l >> 3) & 7u),
              k = 8 * (int)(tile / (D.tx * D.ty)) + (int)(l >> 6);
    const uint8_t t = gen_type(i, j, k, D, surface, sph, nsph);
    type[s] = t;
    float bv = 0.0f;
    if (t == kFluid) {
        float div = 0.0f;
        for (int c = 0; c < 3; ++c)
            div += gen_face(c, i + (c == 0), j + (c == 1), k + (c == 2), D, surface, sph, nsph, imp, nimp, gdt) -
                   gen_face(c, i, j, k, D, surface, sph, nsph, imp, nimp, gdt);
        bv = -div;
    }
    b[s] = bv;
}
// tiles holding at least one fluid cell
__global__ void nat_mark_fluid_tiles_kernel(const uint8_t* __restrict__ type, uint8_t* __restrict__ flags, uint64_t nslots) {
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nslots && type[s] == kFluid) flags[s >> 9] = 1;
}
// the solution x + xg into x on the fluid cells of the last solve, 0
// elsewhere; xg = 0 (the pressure buffer a caller reads)
__global__ void nat_fold_pressure_kernel(double* __restrict__ x, float* __restrict__ xg, const uint8_t* __restrict__ cell,
                                         uint64_t nslots) {
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    x[s] = (cell[s] & kCellFluid) ? x[s] + (double)xg[s] : 0.0;
    xg[s] = 0.0f;
}
// x-fastest linear array -> tile-blocked slots (and back)
__global__ void nat_lin_tiles_f32_kernel(const float* __restrict__ src, float* __restrict__ dst, NatDims D, int to_tiles) {
    const uint64_t id = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nc = (uint64_t)D.nx * D.ny * D.nz;
    if (id >= nc) return;
    const int i = (int)(id % D.nx), j = (int)((id / D.nx) % D.ny), k = (int)(id / ((uint64_t)D.nx * D.ny));
    const uint32_t s = nslot(i, j, k, D);
    if (to_tiles) dst[s] = src[id];
    else dst[id] = src[s];
}

// solution x + xg of the fluid cells in x-fastest order (0 elsewhere)
__global__ void nat_solution_lin_kernel(const double* __restrict__ x, const float* __restrict__ xg,
                                        const uint8_t* __restrict__ cell, NatDims D, double* __restrict__ out) {
    const uint64_t id = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nc = (uint64_t)D.nx * D.ny * D.nz;
    if (id >= nc) return;
    const int i = (int)(id % D.nx), j = (int)((id / D.nx) % D.ny), k = (int)(id / ((uint64_t)D.nx * D.ny));
    const uint32_t s = nslot(i, j, k, D);
    out[id] = (cell[s] & kCellFluid) ? x[s] + (double)xg[s] : 0.0;
}

// tiles touched by the stencils of occupied tiles: 3x3x3 dilation
__global__ void nat_dilate_kernel(const uint32_t* __restrict__ tile_keys, const uint32_t* __restrict__ d_ntiles, NatDims D,
                                  uint8_t* __restrict__ flags) {
    const uint32_t ntiles = *d_ntiles;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x) {
        uint32_t key = tile_keys[t];
        int tx = key % D.tx, ty = (key / D.tx) % D.ty, tz = key / (D.tx * D.ty);
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    int a = tx + dx, b = ty + dy, c = tz + dz;
                    if (a < 0 || b < 0 || c < 0 || a >= D.tx || b >= D.ty || c >= D.tz) continue;
                    flags[a + D.tx * (b + D.ty * c)] = 1;
                }
    }
}

// single-CTA compaction of tile flags into a list (ascending tile order)
constexpr int kCompactThreads = 1024;
__global__ void __launch_bounds__(kCompactThreads) nat_compact_kernel(const uint8_t* __restrict__ flags, uint32_t ntotal,
                                                                       uint32_t* __restrict__ list, uint32_t* __restrict__ d_count) {
    __shared__ uint32_t sh[kCompactThreads / 32 + 1];
    const uint32_t per = (ntotal + kCompactThreads - 1) / kCompactThreads;
    const uint32_t b0 = threadIdx.x * per, b1 = min(ntotal, b0 + per);
    uint32_t c = 0;
    for (uint32_t i = b0; i < b1; ++i) c += flags[i] ? 1u : 0u;
    uint32_t total;
    uint32_t o = block_exclusive_scan<kCompactThreads>(c, sh, &total);
    for (uint32_t i = b0; i < b1; ++i)
        if (flags[i]) list[o++] = i;
    if (threadIdx.x == 0) *d_count = total;
}

// Segment heads of the sorted tile keys: the sort's last pass leaves
// dense[key] = the index of the first particle with that tile key (kNoHead
// for an empty tile; no scan of head flags, no look-back chain), and one CTA
// lists the occupied tiles in key order -- the order of the sorted segments
// -- with their starts.  It takes the table in chunks staged in shared
// memory by coalesced loads; a thread then counts and writes 8 consecutive
// entries (stored one word of padding per 8, so that a warp's reads fall on
// distinct banks).
constexpr uint32_t kNoHead = 0xFFFFFFFFu;
constexpr int kHcPer = 8;
constexpr uint32_t kHcChunk = (uint32_t)kCompactThreads * kHcPer;
__device__ __forceinline__ uint32_t hc_slot(uint32_t i) { return i + (i >> 3); }
__global__ void __launch_bounds__(kCompactThreads) nat_heads_compact_kernel(const uint32_t* __restrict__ dense,
                                                                            uint32_t ntotal, uint32_t* __restrict__ list,
                                                                            uint32_t* __restrict__ starts,
                                                                            uint32_t* __restrict__ d_count) {
    __shared__ uint32_t sd[kHcChunk + kHcChunk / 8];
    __shared__ uint32_t sh[kCompactThreads / 32 + 1];
    const uint32_t tid = threadIdx.x;
    uint32_t out = 0;
    for (uint32_t c0 = 0; c0 < ntotal; c0 += kHcChunk) {
        const uint32_t m = min(kHcChunk, ntotal - c0);
        uint32_t v[kHcPer];
#pragma unroll
        for (int r = 0; r < kHcPer; ++r) {
            const uint32_t i = tid + r * kCompactThreads;
            v[r] = i < m ? dense[c0 + i] : kNoHead;
        }
#pragma unroll
        for (int r = 0; r < kHcPer; ++r) sd[hc_slot(tid + r * kCompactThreads)] = v[r];
        __syncthreads();
        const uint32_t b0 = tid * kHcPer;
        uint32_t c = 0;
#pragma unroll
        for (int r = 0; r < kHcPer; ++r) {
            v[r] = sd[hc_slot(b0 + r)];
            c += v[r] != kNoHead ? 1u : 0u;
        }
        uint32_t total;
        uint32_t o = out + block_exclusive_scan<kCompactThreads>(c, sh, &total);
#pragma unroll
        for (int r = 0; r < kHcPer; ++r)
            if (v[r] != kNoHead) {
                list[o] = c0 + b0 + r;
                starts[o] = v[r];
                ++o;
            }
        out += total;
        __syncthreads();  // the next chunk overwrites sd and sh
    }
    if (tid == 0) *d_count = out;
}

// solid mask (tile-blocked) onto the cell types
__global__ void nat_apply_solids_kernel(const uint8_t* __restrict__ solid, uint8_t* __restrict__ type, uint64_t nslots) {
    uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nslots && solid[s]) type[s] = kSolid;
}

// linear (x fastest) mask -> tile-blocked
__global__ void nat_mask_to_tiles_kernel(const uint8_t* __restrict__ lin, NatDims D, uint8_t* __restrict__ tiled) {
    uint64_t id = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t nc = (uint64_t)D.nx * D.ny * D.nz;
    if (id >= nc) return;
    int i = (int)(id % D.nx), j = (int)((id / D.nx) % D.ny), k = (int)(id / ((uint64_t)D.nx * D.ny));
    tiled[nslot(i, j, k, D)] = lin[id];
}

// -------------------------------------------- normalise + classify faces
// 512 threads per tile, one per slot.  Momentum/weight -> velocity; the
// pre-gravity value is the FLIP "old" grid; faces touching a solid cell are
// zero; faces touching a fluid cell receive gravity.
__global__ void __launch_bounds__(512) nat_normalize_kernel(const uint32_t* __restrict__ tiles, const uint32_t* __restrict__ d_count,
                                                             NatDims D, float gdt, float* __restrict__ mu, float* __restrict__ mv,
                                                             float* __restrict__ mw, const float* __restrict__ wu,
                                                             const float* __restrict__ wv, const float* __restrict__ ww,
                                                             float* __restrict__ ou, float* __restrict__ ov,
                                                             float* __restrict__ ow, const uint8_t* __restrict__ type,
                                                             float3 usolid, float* __restrict__ lu, float* __restrict__ lv,
                                                             float* __restrict__ lw, float* __restrict__ lou,
                                                             float* __restrict__ lov, float* __restrict__ low,
                                                             const float* __restrict__ gdt_p) {
    const uint32_t cnt = *d_count;
    if (gdt_p) gdt = *gdt_p;
    const float us[3] = {usolid.x, usolid.y, usolid.z};
    float* m[3] = {mu, mv, mw};
    const float* w[3] = {wu, wv, ww};
    float* o[3] = {ou, ov, ow};
    float* L[3] = {lu, lv, lw};
    float* LO[3] = {lou, lov, low};
    const int li = threadIdx.x & 7, lj = (threadIdx.x >> 3) & 7, lk = threadIdx.x >> 6;
    for (uint32_t t = blockIdx.x; t < cnt; t += gridDim.x) {
        const uint32_t key = tiles[t];
        const int i = 8 * (key % D.tx) + li, j = 8 * ((key / D.tx) % D.ty) + lj, k = 8 * (key / (D.tx * D.ty)) + lk;
        const uint32_t s = (key << 9) | threadIdx.x;
        const uint32_t lin = (uint32_t)i + (uint32_t)D.nx * ((uint32_t)j + (uint32_t)D.ny * (uint32_t)k);
        const uint8_t tb = type[s];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float wt = w[c][s];
            float val = wt > 0.0f ? __fdiv_rn(m[c][s], wt) : 0.0f;
            o[c][s] = val;
            if (LO[c]) LO[c][lin] = val;
            uint8_t ta = nat_type(type, i - (c == 0), j - (c == 1), k - (c == 2), D);
            // wall faces and faces between two solids 0; a face between a
            // solid and a non-solid cell moves with the solid
            const bool wall = (c == 0 ? i : (c == 1 ? j : k)) == 0;
            if (ta == kSolid || tb == kSolid) val = (!wall && ((ta == kSolid) != (tb == kSolid))) ? us[c] : 0.0f;
            else if (c == 1 && (ta == kFluid || tb == kFluid)) val += gdt;
            m[c][s] = val;
            if (L[c]) L[c][lin] = val;
        }
    }
}

// ---------------------------------------------------------------- PCG
// Jacobi-preconditioned CG on A phi = -div over fluid cells: A has the
// number of non-solid neighbours on the diagonal and -1 for each fluid
// neighbour (air neighbours are Dirichlet zero, solid ones Neumann).

template <int NV>
__device__ __forceinline__ bool last_block_reduce(double (&v)[NV], double* partials, unsigned int* ticket, double* sh,
                                                  double (&out)[NV]) {
    return last_block_reduce_n<NV, 512>(v, partials, ticket, sh, out);
}

#define NAT_TILE_LOOP_BEGIN                                                                   \
    const int li = threadIdx.x & 7, lj = (threadIdx.x >> 3) & 7, lk = threadIdx.x >> 6;      \
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {                               \
        const uint32_t key = tiles[t];                                                        \
        const int i = 8 * (key % D.tx) + li, j = 8 * ((key / D.tx) % D.ty) + lj,             \
                  k = 8 * (key / (D.tx * D.ty)) + lk;                                         \
        const uint32_t s = (key << 9) | threadIdx.x;                                          \
        (void)i; (void)j; (void)k;
#define NAT_TILE_LOOP_END }

// 1/d for d = 0..7 (0 for d = 0), the Jacobi inverse diagonal
__constant__ float kJacobiInv[8] = {0.0f, 1.0f, 0.5f, 1.0f / 3.0f, 0.25f, 0.2f, 1.0f / 6.0f, 1.0f / 7.0f};
__device__ __forceinline__ float jacobi_inv(uint8_t c) {
    uint32_t d = c & 7u;
    return d ? __frcp_rn((float)d) : 0.0f;
}
// the same values from a per-CTA shared copy (no MUFU, no divergence on the constant bank)
__device__ __forceinline__ float jacobi_inv_s(const float* tab, uint8_t c) { return tab[c & 7u]; }

// divergence -> b = -div; cell codes; x = 0, r = b, p = 0 (the first
// direction update turns p into D^-1 r)
// cell_prev (warm start): the previous solve's cell codes; x starts from the
// previous solution (x + xg) on cells that are fluid in both solves, 0
// elsewhere, and pcg_warm_kernel then replaces r = b by b - A x
// W (the plain solve's scaled form): r holds w = D^-1 r (0 where d = 0: a
// fluid cell walled in by solids has an empty row of A), and the tiles walked
// are the dilated list, so that w and both direction buffers are also zero on
// the non-fluid cells around the fluid: the matvec then reads its halo
// without the neighbours' cell codes
template <bool W>
__global__ void __launch_bounds__(512, 4) pcg_init_kernel(const uint32_t* __restrict__ tiles, const uint32_t* __restrict__ d_ntiles,
                                                        NatDims D, const float* __restrict__ u, const float* __restrict__ v,
                                                        const float* __restrict__ w, const uint8_t* __restrict__ type,
                                                        const uint8_t* __restrict__ cell_prev, PcgBuffers B) {
    __shared__ double sh[32];
    const uint32_t ntiles = *d_ntiles;
    const bool warm = cell_prev && (!B.warm_ok || *B.warm_ok);
    double bb = 0.0, rz = 0.0, nf = 0.0;
    NAT_TILE_LOOP_BEGIN
    float b = 0.0f;
    uint8_t code = 0;
    if (type[s] == kFluid) {
        if (u) {
            float up = (i + 1 < D.nx) ? u[nslot(i + 1, j, k, D)] : 0.0f;
            float vp = (j + 1 < D.ny) ? v[nslot(i, j + 1, k, D)] : 0.0f;
            float wp = (k + 1 < D.nz) ? w[nslot(i, j, k + 1, D)] : 0.0f;
            float div = ((up - u[s]) + (vp - v[s])) + (wp - w[s]);
            b = -div;
        } else {
            b = B.b[s];
        }
        nf += 1.0;
        uint32_t dcount = 0;
        dcount += nat_type(type, i - 1, j, k, D) != kSolid;
        dcount += nat_type(type, i + 1, j, k, D) != kSolid;
        dcount += nat_type(type, i, j - 1, k, D) != kSolid;
        dcount += nat_type(type, i, j + 1, k, D) != kSolid;
        dcount += nat_type(type, i, j, k - 1, D) != kSolid;
        dcount += nat_type(type, i, j, k + 1, D) != kSolid;
        code = (uint8_t)(kCellFluid | dcount);
    }
    B.cell[s] = code;
    B.b[s] = b;
    double x0 = 0.0;
    if (warm && (code & kCellFluid) && (cell_prev[s] & kCellFluid)) x0 = B.x[s] + (double)B.xg[s];
    B.x[s] = x0;
    B.xg[s] = 0.0f;
    const float z = b * jacobi_inv(code);
    B.r[s] = W ? ((code & 7u) ? __fdiv_rn(b, (float)(code & 7u)) : 0.0f) : b;
    B.p0[s] = 0.0f;
    if (W) B.p1[s] = 0.0f;
    bb += (double)b * (double)b;
    rz += (double)b * (double)z;
    NAT_TILE_LOOP_END
    double vals[3] = {bb, rz, nf}, out[3];
    if (last_block_reduce<3>(vals, B.partials, &B.st->ticket, sh, out) && threadIdx.x == 0) {
        PcgState* st = B.st;
        st->bb = out[0];
        st->rr_check = out[0];
        st->nfluid = out[2];
        st->inv_s = out[0] > 0.0 ? (float)(1.0 / sqrt(out[0] / fmax(out[2], 1.0))) : 1.0f;
        st->zq = 0.0;
        st->rz = out[1];
        st->rz_prev = out[1];
        st->rr = out[0];
        st->beta = 0.0;
        st->pcur = 0;
        st->flush = 0;
        st->iter = 0;
        st->pending = 0;
        st->done = (out[0] == 0.0) ? 1 : 0;
        st->halt = st->done;
    }
}

// p' of one cell: D^-1 r + beta p (Jacobi PCG) on fluid cells, 0 elsewhere
__device__ __forceinline__ float dir_value(const float* tab, uint8_t c, float r, float p, float beta) {
    return (c & kCellFluid) ? fmaf(beta, p, r * jacobi_inv_s(tab, c)) : 0.0f;
}
// flexible PCG: the preconditioned residual z is given
__device__ __forceinline__ float dir_value_z(uint8_t c, float z, float p, float beta) {
    return (c & kCellFluid) ? fmaf(beta, p, z) : 0.0f;
}

// The halo cell a thread loads, as constants of the thread: face f = tid/64
// (0..5: -x, +x, -y, +y, -z, +z; 6, 7: none), the neighbour tile's key
// offset, the cell's slot inside that tile, and the tile-coordinate test for
// the neighbour to exist (packed coordinates: 10 bits per axis).
struct HaloSlot {
    int face;
    int delta;     // neighbour key = key + delta
    uint32_t hl;   // slot within the neighbour tile
    int shift;     // bit offset of the face's axis in the packed coordinates
    int lim;       // -1: need coordinate > 0; else need coordinate < lim
    int hx, hy, hz;  // offsets from the tile origin, -1..8 (shared-memory box)
};
__device__ __forceinline__ HaloSlot halo_slot(int tid, const NatDims& D) {
    HaloSlot h;
    h.face = tid >> 6;
    const int e0 = tid & 7, e1 = (tid >> 3) & 7;
    h.delta = 0; h.hl = 0; h.shift = 0; h.lim = -1; h.hx = h.hy = h.hz = 0;
    switch (h.face) {
    case 0: h.delta = -1; h.hl = 7 + 8 * e0 + 64 * e1; h.shift = 0; h.lim = -1; h.hx = -1; h.hy = e0; h.hz = e1; break;
    case 1: h.delta = 1; h.hl = 8 * e0 + 64 * e1; h.shift = 0; h.lim = D.tx - 1; h.hx = 8; h.hy = e0; h.hz = e1; break;
    case 2: h.delta = -D.tx; h.hl = e0 + 56 + 64 * e1; h.shift = 10; h.lim = -1; h.hx = e0; h.hy = -1; h.hz = e1; break;
    case 3: h.delta = D.tx; h.hl = e0 + 64 * e1; h.shift = 10; h.lim = D.ty - 1; h.hx = e0; h.hy = 8; h.hz = e1; break;
    case 4: h.delta = -D.tx * D.ty; h.hl = e0 + 8 * e1 + 448; h.shift = 20; h.lim = -1; h.hx = e0; h.hy = e1; h.hz = -1; break;
    case 5: h.delta = D.tx * D.ty; h.hl = e0 + 8 * e1; h.shift = 20; h.lim = D.tz - 1; h.hx = e0; h.hy = e1; h.hz = 8; break;
    default: break;
    }
    return h;
}
// slot of the thread's halo cell for the tile (key, packed coordinates tc), or -1
__device__ __forceinline__ int64_t halo_at(const HaloSlot& h, uint32_t key, uint32_t tc) {
    if (h.face >= 6) return -1;
    const int c = (int)((tc >> h.shift) & 1023u);
    const bool ok = h.lim < 0 ? c > 0 : c < h.lim;
    if (!ok) return -1;
    return (int64_t)((((uint32_t)((int)key + h.delta)) << 9) | h.hl);
}

// ---------------------------------------------------------------------------
// Fused direction update + matvec: p' = D^-1 r + beta p (or z + beta p for
// flexible CG) for a tile and its one-cell halo into shared memory (the halo
// cells belong to neighbouring tiles, which compute the same values for
// themselves), then q = A p' from shared memory, and p'.q.  p' goes to the
// other p buffer because neighbouring tiles still read p.  After a
// true-residual check this kernel also folds xg into x.
// Vectorised: a CTA of 512 threads runs four
// independent groups of 128; each group walks its own tiles and syncs on its
// own named barrier.  A thread owns four consecutive x-cells of one (y, z) row
// (float4 loads and stores) and three of the tile's 384 halo cells.  The
// tile's p' goes to a 10 x 10 x 24-float shared box (rows padded so that
// x = 0 and x = 4 start on 16 bytes, x = -1 .. 8 at row offsets 3 .. 12, and
// so that the 16-byte row accesses of a quarter warp, four consecutive rows,
// fall on distinct banks),
// two boxes per group alternating per tile, and the stencil reads its y and
// z neighbours as 16-byte rows.  Loads of the group's next tile are issued
// before the current tile's barrier.
constexpr int kDm4Groups = 4;
constexpr int kDm4Blocks = 296;  // 148 SMs x 2 CTAs
constexpr int kBoxRow = 24;  // 96 B rows: four consecutive rows start 8 banks apart
constexpr int kBoxFloats = 10 * 10 * kBoxRow;
__device__ __forceinline__ int box_at(int x, int y, int z) { return ((z + 1) * 10 + (y + 1)) * kBoxRow + x + 4; }

struct Dm4Loads {
    uint32_t key;
    float4 r, p;
    uint32_t c;
    float hr[3], hp[3];
    uint32_t hc;  // the three halo codes, a byte each
};

// what the direction update starts from:
//   kDmJacobi  r, p' = D^-1 r + beta p on fluid cells (codes of the tile and halo);
//   kDmFlex    z (flexible CG, the preconditioned residual given), p' = z + beta p on fluid cells;
//   kDmScaled  w = D^-1 r, zero off the fluid like p on the dilated tiles, p' = w + beta p: the
//              halo needs no cell codes (the plain solve)
enum DmMode { kDmJacobi = 0, kDmFlex = 1, kDmScaled = 2 };
template <int kMode>
__device__ __forceinline__ float dir1(const float* tab, uint8_t c, float r, float p, float beta) {
    if (kMode == kDmScaled) return fmaf(beta, p, r);
    return kMode == kDmFlex ? dir_value_z(c, r, p, beta) : dir_value(tab, c, r, p, beta);
}
template <int kMode>
__device__ __forceinline__ float4 dir4(const float* tab, uint32_t c4, float4 r, float4 p, float beta) {
    float4 o;
    o.x = dir1<kMode>(tab, (uint8_t)c4, r.x, p.x, beta);
    o.y = dir1<kMode>(tab, (uint8_t)(c4 >> 8), r.y, p.y, beta);
    o.z = dir1<kMode>(tab, (uint8_t)(c4 >> 16), r.z, p.z, beta);
    o.w = dir1<kMode>(tab, (uint8_t)(c4 >> 24), r.w, p.w, beta);
    return o;
}

constexpr int kDm4Smem = kDm4Groups * 2 * kBoxFloats * (int)sizeof(float);
template <int kMode>
__global__ void __launch_bounds__(512, 2) pcg_dirmatvec4_kernel(const uint32_t* __restrict__ tiles,
                                                                 const uint32_t* __restrict__ tcoord,
                                                                 const uint32_t* __restrict__ d_ntiles, NatDims D,
                                                                 const float* __restrict__ r, float* p0, float* p1,
                                                                 const uint8_t* __restrict__ cell, float* __restrict__ q,
                                                                 double* __restrict__ x, float* __restrict__ xg,
                                                                 PcgState* st, double* partials) {
    if (st->done || st->pending) return;
    const float* __restrict__ p = st->pcur ? p1 : p0;
    float* __restrict__ pn = st->pcur ? p0 : p1;
    extern __shared__ __align__(16) float dm4_box[];  // [groups][2][kBoxFloats], dynamic (51 KB)
    __shared__ double sh[32];
    __shared__ float tab[8];
    __shared__ int fdelta[6], flim[6];
    if (threadIdx.x < 8) tab[threadIdx.x] = kJacobiInv[threadIdx.x];
    if (threadIdx.x < 6) {
        const int f = threadIdx.x;
        const int d = f < 2 ? 1 : (f < 4 ? D.tx : D.tx * D.ty);
        const int T = f < 2 ? D.tx : (f < 4 ? D.ty : D.tz);
        fdelta[f] = (f & 1) ? d : -d;
        flim[f] = (f & 1) ? T - 1 : -1;
    }
    __syncthreads();
    const uint32_t ntiles = *d_ntiles;
    const float beta = (float)st->beta;
    const bool flush = st->flush != 0;
    const int g = threadIdx.x >> 7, u = threadIdx.x & 127;
    const int row = u >> 1, half = u & 1;
    const int cy = row & 7, cz = row >> 3, cx = 4 * half;
    const uint32_t lo = (uint32_t)(cx + 8 * cy + 64 * cz);
    const int bo = box_at(cx, cy, cz);
    // halo cells u, u+128, u+256: face h/64, (e0, e1) = in-face position
    uint32_t hA[3];  // face | slot-in-neighbour << 3 | box index << 12
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int h = u + 128 * k, f = h >> 6, e0 = h & 7, e1 = (h >> 3) & 7;
        int hl = 0, bxi = 0;
        switch (f) {
        case 0: hl = 7 + 8 * e0 + 64 * e1; bxi = box_at(-1, e0, e1); break;
        case 1: hl = 8 * e0 + 64 * e1; bxi = box_at(8, e0, e1); break;
        case 2: hl = e0 + 56 + 64 * e1; bxi = box_at(e0, -1, e1); break;
        case 3: hl = e0 + 64 * e1; bxi = box_at(e0, 8, e1); break;
        case 4: hl = e0 + 8 * e1 + 448; bxi = box_at(e0, e1, -1); break;
        default: hl = e0 + 8 * e1; bxi = box_at(e0, e1, 8); break;
        }
        hA[k] = (uint32_t)f | ((uint32_t)hl << 3) | ((uint32_t)bxi << 12);
    }
    const uint32_t stride = gridDim.x * kDm4Groups;
    auto load = [&](Dm4Loads& L, uint32_t t) {
        const uint32_t key = tiles[t];
        const uint32_t tc = tcoord[t];
        L.key = key;
        const uint32_t s = (key << 9) | lo;
        L.r = *reinterpret_cast<const float4*>(r + s);
        L.p = *reinterpret_cast<const float4*>(p + s);
        L.c = *reinterpret_cast<const uint32_t*>(cell + s);
        L.hc = 0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int f = (int)(hA[k] & 7u);
            const int cc = (int)((tc >> (10 * (f >> 1))) & 1023u);
            const int lim = flim[f];
            const bool ok = lim < 0 ? cc > 0 : cc < lim;
            L.hr[k] = 0.0f;
            L.hp[k] = 0.0f;
            if (ok) {
                const uint32_t sn = (((uint32_t)((int)key + fdelta[f])) << 9) | ((hA[k] >> 3) & 511u);
                L.hr[k] = r[sn];
                L.hp[k] = p[sn];
                if (kMode != kDmScaled) L.hc |= (uint32_t)cell[sn] << (8 * k);
            }
        }
    };
    double pq = 0.0;
    Dm4Loads cur;
    uint32_t t = (uint32_t)(blockIdx.x * kDm4Groups + g);
    if (t < ntiles) load(cur, t);
    for (int it = 0; t < ntiles; t += stride, ++it) {
        float* Bx = dm4_box + (2 * g + (it & 1)) * kBoxFloats;
        const uint32_t s = (cur.key << 9) | lo;
        const float4 pc = dir4<kMode>(tab, cur.c, cur.r, cur.p, beta);
        *reinterpret_cast<float4*>(Bx + bo) = pc;
        *reinterpret_cast<float4*>(pn + s) = pc;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const uint8_t hc = (uint8_t)(cur.hc >> (8 * k));
            Bx[hA[k] >> 12] = dir1<kMode>(tab, hc, cur.hr[k], cur.hp[k], beta);
        }
        if (flush && cur.c) {
            const float* gv = xg + s;
#pragma unroll
            for (int m = 0; m < 4; ++m)
                if ((cur.c >> (8 * m)) & kCellFluid) {
                    x[s + m] += (double)gv[m];
                    xg[s + m] = 0.0f;
                }
        }
        Dm4Loads nxt;
        const uint32_t tn = t + stride;
        if (tn < ntiles) load(nxt, tn);
        asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(128) : "memory");
        const float left = Bx[bo - 1], right = Bx[bo + 4];
        const float4 ym = *reinterpret_cast<const float4*>(Bx + bo - kBoxRow);
        const float4 yp = *reinterpret_cast<const float4*>(Bx + bo + kBoxRow);
        const float4 zm = *reinterpret_cast<const float4*>(Bx + bo - 10 * kBoxRow);
        const float4 zp = *reinterpret_cast<const float4*>(Bx + bo + 10 * kBoxRow);
        const float xl[4] = {left, pc.x, pc.y, pc.z}, xr[4] = {pc.y, pc.z, pc.w, right};
        const float yl[4] = {ym.x, ym.y, ym.z, ym.w}, yr[4] = {yp.x, yp.y, yp.z, yp.w};
        const float zl[4] = {zm.x, zm.y, zm.z, zm.w}, zr[4] = {zp.x, zp.y, zp.z, zp.w};
        const float pv[4] = {pc.x, pc.y, pc.z, pc.w};
        float qv[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const uint8_t c = (uint8_t)(cur.c >> (8 * m));
            float qc = 0.0f;
            if (c & kCellFluid) {
                const float sum = ((xl[m] + xr[m]) + (yl[m] + yr[m])) + (zl[m] + zr[m]);
                qc = fmaf((float)(c & 7u), pv[m], -sum);
            }
            qv[m] = qc;
            pq += (double)pv[m] * (double)qc;
        }
        *reinterpret_cast<float4*>(q + s) = make_float4(qv[0], qv[1], qv[2], qv[3]);
        cur = nxt;
    }
    double vals[1] = {pq}, out[1];
    if (last_block_reduce<1>(vals, partials, &st->ticket, sh, out) && threadIdx.x == 0) {
        st->pq = out[0];
        st->flush = 0;
        if (out[0] > 0.0) st->alpha = st->rz / out[0];
        else { st->alpha = 0.0; st->done = 3; }  // breakdown
    }
}

// xg += alpha p, r -= alpha q, partial r.r and r.z; eight cells per thread
// per round (two 16-byte quads per array, all loads issued before use)
// W: r4 holds w = D^-1 r: w -= a D^-1 q, r.r = sum (d w)^2, r.z = sum d w^2
template <bool W>
__device__ __forceinline__ void upd_quad(const float* tab, uint32_t c4, const float4& p4, const float4& q4, float4& r4,
                                         float4& g4, float a, double& rr, double& rz) {
    float* rv = &r4.x;
    float* gv = &g4.x;
    const float* pv = &p4.x;
    const float* qv = &q4.x;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const uint8_t c = (uint8_t)(c4 >> (8 * m));
        if (!(c & kCellFluid)) continue;
        gv[m] = fmaf(a, pv[m], gv[m]);
        if (W) {
            const float d = (float)(c & 7u);
            const float wn = fmaf(-a, qv[m] * jacobi_inv_s(tab, c), rv[m]);
            rv[m] = wn;
            const float rs = d * wn;
            rr += (double)rs * (double)rs;
            rz += (double)rs * (double)wn;
        } else {
            const float rs = fmaf(-a, qv[m], rv[m]);
            rv[m] = rs;
            const float z = rs * jacobi_inv_s(tab, c);
            rr += (double)rs * (double)rs;
            rz += (double)rs * (double)z;
        }
    }
}

// A warp takes a unit of kUpdQuads x 32 quads (half a tile): each lane
// issues all 5 x kUpdQuads loads of its quads before using any of them, and
// the next unit's tile key is loaded one unit ahead.
constexpr int kUpdThreads = 256;
constexpr int kUpdQuads = 2;                    // quads per lane and unit
constexpr int kUpdUnits = 128 / (32 * kUpdQuads);  // units per tile
template <bool W>
__global__ void __launch_bounds__(kUpdThreads, 4) pcg_update_kernel(const uint32_t* __restrict__ tiles,
                                                                     const uint32_t* __restrict__ d_ntiles, NatDims D,
                                                                     float* __restrict__ xg, float* __restrict__ r,
                                                                     const float* p0, const float* p1,
                                                                     const float* __restrict__ q,
                                                                     const uint8_t* __restrict__ cell, PcgState* st,
                                                                     double* partials) {
    if (st->done || st->pending) return;
    const float* __restrict__ p = st->pcur ? p0 : p1;  // the direction the matvec just wrote
    __shared__ double sh[32];
    __shared__ float tab[8];
    if (threadIdx.x < 8) tab[threadIdx.x] = kJacobiInv[threadIdx.x];
    __syncthreads();
    const uint32_t nunits = *d_ntiles * kUpdUnits;
    const float a = (float)st->alpha;
    const int lane = threadIdx.x & 31;
    const uint32_t nwarps = gridDim.x * (kUpdThreads / 32);
    uint32_t w = blockIdx.x * (kUpdThreads / 32) + (threadIdx.x >> 5);
    double rr = 0.0, rz = 0.0;
    uint32_t key = w < nunits ? tiles[w / kUpdUnits] : 0u;
    for (; w < nunits; w += nwarps) {
        const uint32_t wn = w + nwarps;
        const uint32_t key_next = wn < nunits ? tiles[wn / kUpdUnits] : 0u;
        const uint32_t qbase = (w % kUpdUnits) * (32 * kUpdQuads) + lane;
        uint32_t c[kUpdQuads];
        float4 pv[kUpdQuads], qv[kUpdQuads], rv[kUpdQuads], gv[kUpdQuads];
#pragma unroll
        for (int m = 0; m < kUpdQuads; ++m) {
            const uint32_t s = (key << 9) | ((qbase + 32 * m) << 2);
            c[m] = *reinterpret_cast<const uint32_t*>(cell + s);
            pv[m] = *reinterpret_cast<const float4*>(p + s);
            qv[m] = *reinterpret_cast<const float4*>(q + s);
            rv[m] = *reinterpret_cast<const float4*>(r + s);
            gv[m] = *reinterpret_cast<const float4*>(xg + s);
        }
#pragma unroll
        for (int m = 0; m < kUpdQuads; ++m) {
            if (!c[m]) continue;
            const uint32_t s = (key << 9) | ((qbase + 32 * m) << 2);
            upd_quad<W>(tab, c[m], pv[m], qv[m], rv[m], gv[m], a, rr, rz);
            *reinterpret_cast<float4*>(r + s) = rv[m];
            *reinterpret_cast<float4*>(xg + s) = gv[m];
        }
        key = key_next;
    }
    double vals[2] = {rr, rz}, out[2];
    if (last_block_reduce_n<2, kUpdThreads>(vals, partials, &st->ticket, sh, out) && threadIdx.x == 0) {
        st->iter += 1;
        st->pcur ^= 1;
        st->rr = out[0];
        if (!st->flexible) {
            st->rz_prev = st->rz;
            st->rz = out[1];
            st->beta = st->rz / st->rz_prev;
        }
        st->inv_s = out[0] > 0.0 ? (float)(1.0 / sqrt(out[0] / fmax(st->nfluid, 1.0))) : 1.0f;
        if (out[0] <= st->tol2 * st->bb) st->pending = 1;  // confirm with the true residual
        else if (st->iter >= st->max_iter) st->done = 2;
        st->halt = st->done || st->pending;
    }
}

// true residual r = b - A (x + xg) in FP64 at the end of a launch chunk: when
// the recursive residual claimed convergence, or every true_every
// iterations.  Replaces r, decides convergence on the true value and asks
// the next direction kernel to fold xg into x.  The FP64 solution of the tile
// and its halo is staged in shared memory like the matvec.
template <bool W>
__global__ void __launch_bounds__(512, 4) pcg_check_kernel(const uint32_t* __restrict__ tiles,
                                                            const uint32_t* __restrict__ tcoord,
                                                            const uint32_t* __restrict__ d_ntiles, NatDims D,
                                                            const double* __restrict__ x, const float* __restrict__ xg,
                                                            const float* __restrict__ bv, float* __restrict__ r,
                                                            const uint8_t* __restrict__ cell, PcgState* st,
                                                            double* partials) {
    if (st->done) return;
    if (!st->pending && (st->true_every <= 0 || st->iter < st->next_check)) return;
    __shared__ double X[1000];
    __shared__ double sh[32];
    const uint32_t ntiles = *d_ntiles;
    const int tid = threadIdx.x;
    const int li = tid & 7, lj = (tid >> 3) & 7, lk = tid >> 6;
    const int bc = (li + 1) + 10 * ((lj + 1) + 10 * (lk + 1));
    const HaloSlot H = halo_slot(tid, D);
    const int bh = (H.hx + 1) + 10 * ((H.hy + 1) + 10 * (H.hz + 1));
    double rr = 0.0, rz = 0.0;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint32_t key = tiles[t];
        const uint32_t s = (key << 9) | tid;
        const uint8_t c = cell[s];
        const double xs = (c & kCellFluid) ? x[s] + (double)xg[s] : 0.0;
        X[bc] = xs;
        if (H.face < 6) {
            const int64_t sn = halo_at(H, key, tcoord[t]);
            double v = 0.0;
            if (sn >= 0 && (cell[sn] & kCellFluid)) v = x[sn] + (double)xg[sn];
            X[bh] = v;
        }
        __syncthreads();
        if (c & kCellFluid) {
            const double sum = ((X[bc - 1] + X[bc + 1]) + (X[bc - 10] + X[bc + 10])) + (X[bc - 100] + X[bc + 100]);
            const double res = (double)bv[s] - ((double)(c & 7u) * xs - sum);
            rr += res * res;
            if (W) {
                const float ws = (c & 7u) ? (float)(res / (double)(c & 7u)) : 0.0f;
                r[s] = ws;
                rz += (double)(c & 7u) * (double)ws * (double)ws;
            } else {
                const float rs = (float)res;
                r[s] = rs;
                rz += (double)rs * (double)(rs * jacobi_inv(c));
            }
        }
        __syncthreads();
    }
    double vals[2] = {rr, rz}, out[2];
    if (last_block_reduce<2>(vals, partials, &st->ticket, sh, out) && threadIdx.x == 0) {
        st->rr = out[0];
        st->rr_true = out[0];
        st->true_checks += 1;
        st->next_check = st->iter + st->true_every;
        if (out[0] <= st->tol2 * st->bb) {
            st->done = 1;
        } else {
            st->flush = 1;
            if (!st->flexible) {
                st->rz = out[1];
                st->beta = st->rz / st->rz_prev;
            }
            st->inv_s = (float)(1.0 / sqrt(out[0] / fmax(st->nfluid, 1.0)));
            if (st->iter >= st->max_iter) st->done = 2;
            // flexible CG that has stopped converging: the true residual norm
            // fell by less than 10% since the previous check
            if (st->flexible && !st->done && out[0] > kFlexStall * st->rr_check) st->done = 4;
        }
        st->rr_check = out[0];
        st->pending = 0;
        st->halt = st->done;
    }
}

// warm start: r = b - A x in FP64 for the initial guess, r.r and r.z, and
// the state for the first iteration (converged already if |r| <= tol |b|;
// b = 0 gives x = 0)
template <bool W>
__global__ void __launch_bounds__(512, 4) pcg_warm_kernel(const uint32_t* __restrict__ tiles,
                                                           const uint32_t* __restrict__ tcoord,
                                                           const uint32_t* __restrict__ d_ntiles, NatDims D,
                                                           double* __restrict__ x, const float* __restrict__ bv,
                                                           float* __restrict__ r, const uint8_t* __restrict__ cell,
                                                           PcgState* st, double* partials) {
    __shared__ double X[1000];
    __shared__ double sh[32];
    const uint32_t ntiles = *d_ntiles;
    const bool zero = !(st->bb > 0.0);
    const int tid = threadIdx.x;
    const int li = tid & 7, lj = (tid >> 3) & 7, lk = tid >> 6;
    const int bc = (li + 1) + 10 * ((lj + 1) + 10 * (lk + 1));
    const HaloSlot H = halo_slot(tid, D);
    const int bh = (H.hx + 1) + 10 * ((H.hy + 1) + 10 * (H.hz + 1));
    double rr = 0.0, rz = 0.0;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint32_t key = tiles[t];
        const uint32_t s = (key << 9) | tid;
        const uint8_t c = cell[s];
        double xs = (c & kCellFluid) ? x[s] : 0.0;
        if (zero && xs != 0.0) {
            x[s] = 0.0;
            xs = 0.0;
        }
        X[bc] = xs;
        if (H.face < 6) {
            const int64_t sn = halo_at(H, key, tcoord[t]);
            double v = 0.0;
            if (!zero && sn >= 0 && (cell[sn] & kCellFluid)) v = x[sn];
            X[bh] = v;
        }
        __syncthreads();
        if (c & kCellFluid) {
            const double sum = ((X[bc - 1] + X[bc + 1]) + (X[bc - 10] + X[bc + 10])) + (X[bc - 100] + X[bc + 100]);
            const double res = (double)bv[s] - ((double)(c & 7u) * xs - sum);
            rr += res * res;
            if (W) {
                const float ws = (c & 7u) ? (float)(res / (double)(c & 7u)) : 0.0f;
                r[s] = ws;
                rz += (double)(c & 7u) * (double)ws * (double)ws;
            } else {
                const float rs = (float)res;
                r[s] = rs;
                rz += (double)rs * (double)(rs * jacobi_inv(c));
            }
        }
        __syncthreads();
    }
    double vals[2] = {rr, rz}, out[2];
    if (last_block_reduce<2>(vals, partials, &st->ticket, sh, out) && threadIdx.x == 0) {
        st->rr = out[0];
        st->rr_true = out[0];
        st->rz = out[1];
        st->rz_prev = out[1];
        st->beta = 0.0;
        st->inv_s = out[0] > 0.0 ? (float)(1.0 / sqrt(out[0] / fmax(st->nfluid, 1.0))) : 1.0f;
        st->done = (zero || out[0] <= st->tol2 * st->bb) ? 1 : 0;
        st->halt = st->done;
    }
}

// flexible CG (Notay's FCG(1), the same recurrence as Polak-Ribiere PCG)
// with the preconditioner M(r) = N(r) + D^-1 r.  This kernel adds the Jacobi
// term to the network output z in place (jacobi = 1; the multilevel
// preconditioner's z is complete).  The new direction p' = z + beta p
// is A-orthogonal to p for beta = -z.q / p.q (q = A p), and alpha = r.z /
// p'.q' is the exact line search along p' (r is orthogonal to p).  A nonlinear N may give r.z < 0;
// alpha is then negative and the step still minimises the A-norm error along
// p', so only r.z = 0 (no progress possible) or a non-finite value ends the
// solve.  init: beta = 0.
__global__ void __launch_bounds__(512, 4) fpcg_dot_kernel(const uint32_t* __restrict__ tiles,
                                                           const uint32_t* __restrict__ d_ntiles, const float* __restrict__ r,
                                                           float* __restrict__ z, const float* __restrict__ q,
                                                           const uint8_t* __restrict__ cell, int init, int jacobi,
                                                           PcgState* st, double* partials) {
    if (st->halt) return;
    __shared__ double sh[32];
    const uint32_t nquads = *d_ntiles * 128u;
    double rz = 0.0, zq = 0.0;
    for (uint32_t qd = blockIdx.x * 512u + threadIdx.x; qd < nquads; qd += gridDim.x * 512u) {
        const uint32_t s = (tiles[qd >> 7] << 9) | ((qd & 127u) << 2);
        const uint32_t c4 = *reinterpret_cast<const uint32_t*>(cell + s);
        if (!c4) continue;
        const float4 r4 = *reinterpret_cast<const float4*>(r + s);
        float4 z4 = *reinterpret_cast<const float4*>(z + s);
        const float4 q4 = *reinterpret_cast<const float4*>(q + s);
        const float* rv = &r4.x;
        float* zv = &z4.x;
        const float* qv = &q4.x;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const uint8_t c = (uint8_t)(c4 >> (8 * m));
            if (!(c & kCellFluid)) continue;
            const float d = (float)(c & 7u);
            if (jacobi) zv[m] = d > 0.0f ? zv[m] + rv[m] / d : zv[m];  // M(r) = N(r) + D^-1 r
            rz += (double)rv[m] * (double)zv[m];
            zq += (double)zv[m] * (double)qv[m];
        }
        if (jacobi) *reinterpret_cast<float4*>(z + s) = z4;  // else z is unchanged
    }
    double vals[2] = {rz, zq}, out[2];
    if (last_block_reduce<2>(vals, partials, &st->ticket, sh, out) && threadIdx.x == 0) {
        st->beta = init ? 0.0 : (st->pq > 0.0 ? -out[1] / st->pq : 0.0);
        st->rz = out[0];
        st->rz_prev = out[0];
        st->zq = out[1];
        if (out[0] == 0.0 || !isfinite(out[0]) || !isfinite(out[1])) { st->done = 3; st->halt = 1; }
    }
}

// --------------------------------------------------------- projection
__global__ void __launch_bounds__(512) nat_project_kernel(const uint32_t* __restrict__ tiles, const uint32_t* __restrict__ d_count,
                                                           NatDims D, const double* __restrict__ phi, const float* __restrict__ phig,
                                                           const uint8_t* __restrict__ type, float* __restrict__ u,
                                                           float* __restrict__ v, float* __restrict__ w,
                                                           float* __restrict__ lu, float* __restrict__ lv,
                                                           float* __restrict__ lw) {
    const uint32_t ntiles = *d_count;
    float* U[3] = {u, v, w};
    float* L[3] = {lu, lv, lw};
    NAT_TILE_LOOP_BEGIN
    const uint8_t tb = type[s];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        int ia = i - (c == 0), ja = j - (c == 1), ka = k - (c == 2);
        uint8_t ta = nat_type(type, ia, ja, ka, D);
        if (ta == kSolid || tb == kSolid) continue;
        if (ta != kFluid && tb != kFluid) continue;
        double pb = (tb == kFluid) ? phi[s] + (double)phig[s] : 0.0;
        const uint32_t sa = (ta == kFluid) ? nslot(ia, ja, ka, D) : 0u;
        double pa = (ta == kFluid) ? phi[sa] + (double)phig[sa] : 0.0;
        const float nu = U[c][s] - (float)(pb - pa);
        U[c][s] = nu;
        if (L[c]) L[c][(uint32_t)i + (uint32_t)D.nx * ((uint32_t)j + (uint32_t)D.ny * (uint32_t)k)] = nu;
    }
    NAT_TILE_LOOP_END
}

// ------------------------------------------------------- G2P + advect
// One CTA per occupied tile (persistent loop).  The new and old face
// velocities around the tile come into shared memory by TMA: for each of the
// six fields one 16 x 12 x 12 box of its linear (x-fastest) copy, from
// (8tx - 4, 8ty - 2, 8tz - 2) -- x starts on a 16-byte boundary, and the
// two-cell margin in y and z (four and four in x) covers the stencils of
// every particle of the tile and of RK2 midpoints that move less than a cell
// (zero fill outside the grid is the wall value).  The tile's particles then
// sample the boxes: the FLIP/PIC blend of the grid velocity change, the RK2
// midpoint through the new grid (from global memory in the rare case that
// the midpoint's stencil leaves the box), the clamp into the box, the
// reseed of particles that entered an interior solid cell (the native form of
// the reference's moveSolids, engine/particles.cu:674-740: the particle
// returns to its position at the start of the step, which lay outside every
// solid, and takes the solid's velocity), and the tile key of the new
// position for the next step's sort.
constexpr int kG2PThreads = 256;
constexpr int kGBx = 16, kGBy = 12, kGBz = 12;
constexpr int kGBoxN = kGBx * kGBy * kGBz;                    // 2304 floats
constexpr uint32_t kGBoxBytes = kGBoxN * sizeof(float);        // 9216 B
constexpr uint32_t kG2PSmem = 6 * kGBoxBytes + 128;            // six boxes + the mbarrier
constexpr uint32_t kG2PSpinLimit = 1u << 24;

// The stencils of one position: per axis the face-aligned base and weight
// (the component's own axis) and the cell-centred ones (the two others), so
// that the three components and both grids share six nat_axis evaluations.
struct PosStencil {
    int fi[3], ci[3];
    float ff[3], cf[3];
};
__device__ __forceinline__ void pos_stencil(const float (&g)[3], const NatDims& D, PosStencil& S) {
    const int nn[3] = {D.nx, D.ny, D.nz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        nat_axis(g[a], nn[a], S.fi[a], S.ff[a]);
        nat_axis(g[a] - 0.5f, nn[a] - 1, S.ci[a], S.cf[a]);
    }
}
// trilinear interpolation of a 2 x 2 x 2 block of a box (b: its lowest corner)
__device__ __forceinline__ float box_lerp(const float* __restrict__ b, float fx, float fy, float fz) {
    const float c00 = fmaf(fx, b[1] - b[0], b[0]);
    const float c10 = fmaf(fx, b[kGBx + 1] - b[kGBx], b[kGBx]);
    const float c01 = fmaf(fx, b[kGBx * kGBy + 1] - b[kGBx * kGBy], b[kGBx * kGBy]);
    const float c11 = fmaf(fx, b[kGBx * kGBy + kGBx + 1] - b[kGBx * kGBy + kGBx], b[kGBx * kGBy + kGBx]);
    const float c0 = fmaf(fy, c10 - c00, c00), c1 = fmaf(fy, c11 - c01, c01);
    return fmaf(fz, c1 - c0, c0);
}
// component c's stencil from S: base (i0, j0, k0) and weights, and its
// offset in a box of origin (bx0, by0, bz0); false when it leaves the box
__device__ __forceinline__ bool comp_stencil(const PosStencil& S, int c, int bx0, int by0, int bz0, int& i0, int& j0,
                                             int& k0, float& fx, float& fy, float& fz, int& off) {
    i0 = c == 0 ? S.fi[0] : S.ci[0];
    j0 = c == 1 ? S.fi[1] : S.ci[1];
    k0 = c == 2 ? S.fi[2] : S.ci[2];
    fx = c == 0 ? S.ff[0] : S.cf[0];
    fy = c == 1 ? S.ff[1] : S.cf[1];
    fz = c == 2 ? S.ff[2] : S.cf[2];
    const int li = i0 - bx0, lj = j0 - by0, lk = k0 - bz0;
    off = li + kGBx * (lj + kGBy * lk);
    return (unsigned)li < (unsigned)(kGBx - 1) && (unsigned)lj < (unsigned)(kGBy - 1) && (unsigned)lk < (unsigned)(kGBz - 1);
}
// the same interpolation from global memory (wall faces take no weight), for
// a stencil outside the box
__device__ __forceinline__ float nat_sample_at(const float* __restrict__ f, int c, int i0, int j0, int k0, float fx, float fy,
                                               float fz, const NatDims& D) {
    float s = 0.0f;
#pragma unroll
    for (int dk = 0; dk < 2; ++dk)
#pragma unroll
        for (int dj = 0; dj < 2; ++dj)
#pragma unroll
            for (int di = 0; di < 2; ++di) {
                const int i = i0 + di, j = j0 + dj, k = k0 + dk;
                if (nat_wall(c, i, j, k, D)) continue;
                const float w = (di ? fx : 1.0f - fx) * (dj ? fy : 1.0f - fy) * (dk ? fz : 1.0f - fz);
                s = fmaf(w, __ldg(f + nslot(i, j, k, D)), s);
            }
    return s;
}

__global__ void __launch_bounds__(kG2PThreads) nat_g2p_tile_kernel(
    const __grid_constant__ CUtensorMap mu, const __grid_constant__ CUtensorMap mv, const __grid_constant__ CUtensorMap mw,
    const __grid_constant__ CUtensorMap mou, const __grid_constant__ CUtensorMap mov, const __grid_constant__ CUtensorMap mow,
    const uint32_t* __restrict__ tile_keys, const uint32_t* __restrict__ starts, const uint32_t* __restrict__ d_ntiles,
    uint64_t n, NatDims D, float dt, float flip, const float* __restrict__ gu, const float* __restrict__ gv,
    const float* __restrict__ gw, const float* __restrict__ gou, const float* __restrict__ gov,
    const float* __restrict__ gow, const float* px, const float* py, const float* pz, const float* vx,
    const float* vy, const float* vz, float* qx, float* qy, float* qz, float* wx, float* wy, float* wz,
    uint32_t* __restrict__ keys_out, const uint8_t* __restrict__ solid_type, float3 usolid, const float* __restrict__ dt_p,
    uint32_t* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char g2p_smem[];
    float* box = reinterpret_cast<float*>(g2p_smem);  // U u, v, w then O u, v, w
    uint64_t* bar = reinterpret_cast<uint64_t*>(g2p_smem + 6 * kGBoxBytes);
    const CUtensorMap* maps[6] = {&mu, &mv, &mw, &mou, &mov, &mow};
    const float* G[3] = {gu, gv, gw};
    const float* GO[3] = {gou, gov, gow};
    if (threadIdx.x == 0) mbar_init(bar, 1);
    __syncthreads();
    const uint32_t ntiles = *d_ntiles;
    if (dt_p) dt = *dt_p;
    const float o[3] = {D.ox, D.oy, D.oz};
    const int nn[3] = {D.nx, D.ny, D.nz};
    const float eps = 1e-3f * D.h;
    uint32_t parity = 0;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint32_t key = tile_keys[t];
        const int tx = (int)(key % D.tx), ty = (int)((key / D.tx) % D.ty), tz = (int)(key / (D.tx * D.ty));
        const int bx0 = 8 * tx - 4, by0 = 8 * ty - 2, bz0 = 8 * tz - 2;
        if (threadIdx.x == 0) {
            fence_proxy_async_smem();  // the previous tile's reads of the boxes come first
            mbar_expect_tx(bar, 6 * kGBoxBytes);
#pragma unroll
            for (int f = 0; f < 6; ++f) tma_load_3d(box + f * kGBoxN, maps[f], bx0, by0, bz0, bar);
        }
        const uint32_t start = starts[t];
        const uint64_t end = (t + 1 < ntiles) ? starts[t + 1] : n;
        // every thread waits on the copies; the CTA decides together
        if (!__syncthreads_and(mbar_wait_bounded(bar, parity, kG2PSpinLimit))) {
            // the copies never completed: report, wait (bounded) once more so
            // that no copy lands after the CTA has left, and stop
            if (threadIdx.x == 0) atomicOr(err, DEVERR_TMA_TIMEOUT);
            mbar_wait_bounded(bar, parity, kG2PSpinLimit);
            return;
        }
        parity ^= 1u;
        for (uint64_t p = start + threadIdx.x; p < end; p += kG2PThreads) {
            float X[3] = {px[p], py[p], pz[p]};
            float V[3] = {vx[p], vy[p], vz[p]};
            PosStencil S;
            {
                const float g[3] = {nat_grid_coord(X[0], o[0], D.inv_h), nat_grid_coord(X[1], o[1], D.inv_h),
                                    nat_grid_coord(X[2], o[2], D.inv_h)};
                pos_stencil(g, D, S);
            }
            float un[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                // the stencils of a particle of this tile lie inside the box;
                // the global reads only guard against a position the binning
                // did not see.  The new and the old grid share the stencil.
                int i0, j0, k0, off;
                float fx, fy, fz, uo;
                if (comp_stencil(S, c, bx0, by0, bz0, i0, j0, k0, fx, fy, fz, off)) {
                    un[c] = box_lerp(box + c * kGBoxN + off, fx, fy, fz);
                    uo = box_lerp(box + (3 + c) * kGBoxN + off, fx, fy, fz);
                } else {
                    un[c] = nat_sample_at(G[c], c, i0, j0, k0, fx, fy, fz, D);
                    uo = nat_sample_at(GO[c], c, i0, j0, k0, fx, fy, fz, D);
                }
                const float vf = V[c] + (un[c] - uo);
                V[c] = flip * vf + (1.0f - flip) * un[c];
            }
            {
                const float gm[3] = {nat_grid_coord(fmaf(0.5f * dt, un[0], X[0]), o[0], D.inv_h),
                                     nat_grid_coord(fmaf(0.5f * dt, un[1], X[1]), o[1], D.inv_h),
                                     nat_grid_coord(fmaf(0.5f * dt, un[2], X[2]), o[2], D.inv_h)};
                pos_stencil(gm, D, S);
            }
            float Xn[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                int i0, j0, k0, off;
                float fx, fy, fz, um;
                if (comp_stencil(S, c, bx0, by0, bz0, i0, j0, k0, fx, fy, fz, off))
                    um = box_lerp(box + c * kGBoxN + off, fx, fy, fz);
                else
                    um = nat_sample_at(G[c], c, i0, j0, k0, fx, fy, fz, D);
                const float xn = fmaf(dt, um, X[c]);
                const float lo = o[c] + eps, hi = o[c] + (float)nn[c] * D.h - eps;
                Xn[c] = fminf(fmaxf(xn, lo), hi);
            }
            // a particle moved into an interior solid cell goes back to where
            // it started the step (a non-solid cell) and moves with the solid
            if (solid_type &&
                solid_type[nslot(nat_cell(Xn[0], D.ox, D.inv_h, D.nx), nat_cell(Xn[1], D.oy, D.inv_h, D.ny),
                                 nat_cell(Xn[2], D.oz, D.inv_h, D.nz), D)] == kSolid) {
                V[0] = usolid.x; V[1] = usolid.y; V[2] = usolid.z;
            } else {
                X[0] = Xn[0]; X[1] = Xn[1]; X[2] = Xn[2];
            }
            qx[p] = X[0]; qy[p] = X[1]; qz[p] = X[2];
            wx[p] = V[0]; wy[p] = V[1]; wz[p] = V[2];
            if (keys_out) {
                const int ci = nat_cell(X[0], D.ox, D.inv_h, D.nx), cj = nat_cell(X[1], D.oy, D.inv_h, D.ny),
                          ck = nat_cell(X[2], D.oz, D.inv_h, D.nz);
                keys_out[p] = (uint32_t)((ci >> 3) + D.tx * ((cj >> 3) + D.ty * (ck >> 3)));
            }
        }
        __syncthreads();  // every thread is done with the boxes before the next copy
    }
}

// ----------------------------------------------------------- launchers
static inline unsigned nb(uint64_t n, int t) { return (unsigned)((n + t - 1) / t); }

int nat_launch_keys(const float* px, const float* py, const float* pz, uint64_t n, const NatDims& D, uint32_t* keys,
                    cudaStream_t s) {
    if (n) nat_keys_kernel<<<nb(n, 256), 256, 0, s>>>(px, py, pz, n, D, keys);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_gather(const uint32_t* perm, uint64_t n, const float* const* src, float* const* dst, cudaStream_t s) {
    if (n)
        nat_gather_kernel<<<nb(n, 256), 256, 0, s>>>(perm, n, src[0], src[1], src[2], src[3], src[4], src[5], dst[0], dst[1],
                                                     dst[2], dst[3], dst[4], dst[5]);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_p2g(const uint32_t* tile_keys, const uint32_t* starts, const uint32_t* d_ntiles, uint64_t n,
                   const float* const* ps, const float* const* vs, const NatDims& D, float* const* m, float* const* w,
                   uint8_t* type, int grid, cudaStream_t s) {
    constexpr size_t smem = sizeof(P2GCellSmem);
    static bool attr_done = false;
    if (!attr_done) {
        FLIP_CUDA_TRY(cudaFuncSetAttribute(nat_p2g_cells_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr_done = true;
    }
    nat_p2g_cells_kernel<<<grid, kPcThreads, smem, s>>>(tile_keys, starts, d_ntiles, n, ps[0], ps[1], ps[2], vs[0], vs[1],
                                                        vs[2], D, m[0], m[1], m[2], w[0], w[1], w[2], type);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_tile_coords(const uint32_t* tile_keys, const uint32_t* d_ntiles, const NatDims& D, uint32_t* coords,
                           int grid, cudaStream_t s) {
    nat_tile_coords_kernel<<<grid, 256, 0, s>>>(tile_keys, d_ntiles, D, coords);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_poisson_gen(const NatDims& D, float surface, const float4* sph, int nsph, const float* imp, int nimp,
                           float gdt, uint8_t* type, float* b, uint64_t nslots, cudaStream_t s) {
    nat_poisson_gen_kernel<<<nb(nslots, 256), 256, 0, s>>>(D, surface, sph, nsph, imp, nimp, gdt, type, b, nslots);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_fluid_tiles(const uint8_t* type, uint8_t* flags, uint32_t ntiles_total, uint32_t* list, uint32_t* d_count,
                           uint64_t nslots, cudaStream_t s) {
    FLIP_CUDA_TRY(cudaMemsetAsync(flags, 0, ntiles_total, s));
    nat_mark_fluid_tiles_kernel<<<nb(nslots, 256), 256, 0, s>>>(type, flags, nslots);
    nat_compact_kernel<<<1, kCompactThreads, 0, s>>>(flags, ntiles_total, list, d_count);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_segment_heads(const uint32_t* dense, uint32_t ntiles_total, uint32_t* list, uint32_t* starts,
                             uint32_t* d_count, cudaStream_t s) {
    nat_heads_compact_kernel<<<1, kCompactThreads, 0, s>>>(dense, ntiles_total, list, starts, d_count);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_fold_pressure(double* x, float* xg, const uint8_t* cell, uint64_t nslots, cudaStream_t s) {
    nat_fold_pressure_kernel<<<nb(nslots, 256), 256, 0, s>>>(x, xg, cell, nslots);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_lin_tiles_f32(const float* src, float* dst, const NatDims& D, int to_tiles, cudaStream_t s) {
    uint64_t nc = (uint64_t)D.nx * D.ny * D.nz;
    nat_lin_tiles_f32_kernel<<<nb(nc, 256), 256, 0, s>>>(src, dst, D, to_tiles);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_solution_lin(const double* x, const float* xg, const uint8_t* cell, const NatDims& D, double* out,
                            cudaStream_t s) {
    uint64_t nc = (uint64_t)D.nx * D.ny * D.nz;
    nat_solution_lin_kernel<<<nb(nc, 256), 256, 0, s>>>(x, xg, cell, D, out);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_dilate_compact(const uint32_t* tile_keys, const uint32_t* d_ntiles, const NatDims& D, uint8_t* flags,
                              uint32_t* list, uint32_t* d_count, int grid, cudaStream_t s) {
    nat_dilate_kernel<<<grid, 256, 0, s>>>(tile_keys, d_ntiles, D, flags);
    nat_compact_kernel<<<1, kCompactThreads, 0, s>>>(flags, (uint32_t)(D.tx * D.ty * D.tz), list, d_count);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_apply_solids(const uint8_t* solid, uint8_t* type, uint64_t nslots, cudaStream_t s) {
    nat_apply_solids_kernel<<<nb(nslots, 256), 256, 0, s>>>(solid, type, nslots);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_mask_to_tiles(const uint8_t* lin, const NatDims& D, uint8_t* tiled, cudaStream_t s) {
    uint64_t nc = (uint64_t)D.nx * D.ny * D.nz;
    nat_mask_to_tiles_kernel<<<nb(nc, 256), 256, 0, s>>>(lin, D, tiled);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_normalize(const uint32_t* tiles, const uint32_t* d_count, const NatDims& D, float gdt, float* const* m,
                         const float* const* w, float* const* o, const uint8_t* type, float3 usolid, int grid,
                         cudaStream_t s, float* const* lin, float* const* lin_old, const float* gdt_p) {
    float* const nl[3] = {nullptr, nullptr, nullptr};
    float* const* L = lin ? lin : nl;
    float* const* LO = lin_old ? lin_old : nl;
    nat_normalize_kernel<<<grid, 512, 0, s>>>(tiles, d_count, D, gdt, m[0], m[1], m[2], w[0], w[1], w[2], o[0], o[1], o[2],
                                              type, usolid, L[0], L[1], L[2], LO[0], LO[1], LO[2], gdt_p);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_pcg_init(const uint32_t* tiles, const uint32_t* d_ntiles, const NatDims& D, const float* const* U,
                        const uint8_t* type, PcgBuffers& B, cudaStream_t s, const uint8_t* cell_prev) {
    pcg_init_kernel<false><<<kPcgBlocks, 512, 0, s>>>(tiles, d_ntiles, D, U[0], U[1], U[2], type, cell_prev, B);
    if (cell_prev)
        pcg_warm_kernel<false><<<kPcgBlocks, 512, 0, s>>>(tiles, B.tcoord, d_ntiles, D, B.x, B.b, B.r, B.cell, B.st,
                                                          B.partials);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_pcgw_init(const uint32_t* tiles, const uint32_t* d_ntiles, const uint32_t* dil_tiles,
                         const uint32_t* d_ndil, const NatDims& D, const float* const* U, const uint8_t* type,
                         PcgBuffers& B, cudaStream_t s, const uint8_t* cell_prev) {
    pcg_init_kernel<true><<<kPcgBlocks, 512, 0, s>>>(dil_tiles, d_ndil, D, U[0], U[1], U[2], type, cell_prev, B);
    if (cell_prev)
        pcg_warm_kernel<true><<<kPcgBlocks, 512, 0, s>>>(tiles, B.tcoord, d_ntiles, D, B.x, B.b, B.r, B.cell, B.st,
                                                         B.partials);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
// the matvec's 51 KB of shared boxes exceed the default 48 KB: raise the limit once per process
static int dm4_prepare() {
    static bool done = false;
    if (done) return FLIP_OK;
    FLIP_CUDA_TRY(cudaFuncSetAttribute(pcg_dirmatvec4_kernel<kDmJacobi>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDm4Smem));
    FLIP_CUDA_TRY(cudaFuncSetAttribute(pcg_dirmatvec4_kernel<kDmFlex>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDm4Smem));
    FLIP_CUDA_TRY(cudaFuncSetAttribute(pcg_dirmatvec4_kernel<kDmScaled>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDm4Smem));
    done = true;
    return FLIP_OK;
}
int nat_launch_fpcg_direction_update(const uint32_t* tiles, const uint32_t* d_ntiles, const NatDims& D, PcgBuffers& B,
                                     cudaStream_t s) {
    if (int rc = dm4_prepare()) return rc;
    pcg_dirmatvec4_kernel<kDmFlex><<<kDm4Blocks, 512, kDm4Smem, s>>>(tiles, B.tcoord, d_ntiles, D, B.z, B.p0, B.p1, B.cell,
                                                                     B.q, B.x, B.xg, B.st, B.partials);
    pcg_update_kernel<false><<<kPcgUpdateBlocks, kUpdThreads, 0, s>>>(tiles, d_ntiles, D, B.xg, B.r, B.p0, B.p1, B.q,
                                                                      B.cell, B.st, B.partials);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_fpcg_dot(const uint32_t* tiles, const uint32_t* d_ntiles, PcgBuffers& B, int init, cudaStream_t s,
                        int jacobi) {
    fpcg_dot_kernel<<<kPcgBlocks, 512, 0, s>>>(tiles, d_ntiles, B.r, B.z, B.q, B.cell, init, jacobi, B.st, B.partials);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_pcg_iteration(const uint32_t* tiles, const uint32_t* d_ntiles, const NatDims& D, PcgBuffers& B,
                             cudaStream_t s) {
    if (int rc = dm4_prepare()) return rc;
    pcg_dirmatvec4_kernel<kDmJacobi><<<kDm4Blocks, 512, kDm4Smem, s>>>(tiles, B.tcoord, d_ntiles, D, B.r, B.p0, B.p1, B.cell,
                                                                       B.q, B.x, B.xg, B.st, B.partials);
    pcg_update_kernel<false><<<kPcgUpdateBlocks, kUpdThreads, 0, s>>>(tiles, d_ntiles, D, B.xg, B.r, B.p0, B.p1, B.q,
                                                                      B.cell, B.st, B.partials);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_pcgw_iteration(const uint32_t* tiles, const uint32_t* d_ntiles, const NatDims& D, PcgBuffers& B,
                              cudaStream_t s) {
    if (int rc = dm4_prepare()) return rc;
    pcg_dirmatvec4_kernel<kDmScaled><<<kDm4Blocks, 512, kDm4Smem, s>>>(tiles, B.tcoord, d_ntiles, D, B.r, B.p0, B.p1, B.cell,
                                                                       B.q, B.x, B.xg, B.st, B.partials);
    pcg_update_kernel<true><<<kPcgUpdateBlocks, kUpdThreads, 0, s>>>(tiles, d_ntiles, D, B.xg, B.r, B.p0, B.p1, B.q,
                                                                     B.cell, B.st, B.partials);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_pcg_check(const uint32_t* tiles, const uint32_t* d_ntiles, const NatDims& D, PcgBuffers& B,
                         cudaStream_t s) {
    pcg_check_kernel<false><<<kPcgBlocks, 512, 0, s>>>(tiles, B.tcoord, d_ntiles, D, B.x, B.xg, B.b, B.r, B.cell, B.st,
                                                       B.partials);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_pcgw_check(const uint32_t* tiles, const uint32_t* d_ntiles, const NatDims& D, PcgBuffers& B,
                          cudaStream_t s) {
    pcg_check_kernel<true><<<kPcgBlocks, 512, 0, s>>>(tiles, B.tcoord, d_ntiles, D, B.x, B.xg, B.b, B.r, B.cell, B.st,
                                                      B.partials);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
__global__ void pcg_loop_ctl_kernel(cudaGraphConditionalHandle h, PcgState* st, int limit) {
    const int c = ++st->chunks;
    cudaGraphSetConditional(h, (st->done || c >= limit) ? 0u : 1u);
}
int nat_launch_loop_ctl(cudaGraphConditionalHandle h, PcgState* st, int limit, cudaStream_t s) {
    pcg_loop_ctl_kernel<<<1, 1, 0, s>>>(h, st, limit);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
// ------------------------------------------------ solve and frame control
__global__ void pcg_state_init_kernel(PcgState* st, double tol2, int max_iter, int true_every, int flexible) {
    PcgState init{};
    init.tol2 = tol2;
    init.max_iter = max_iter;
    init.true_every = true_every;
    init.next_check = true_every;
    init.flexible = flexible;
    *st = init;
}
int nat_launch_state_init(PcgState* st, double tol, int max_iter, int true_every, int flexible, cudaStream_t s) {
    pcg_state_init_kernel<<<1, 1, 0, s>>>(st, tol * tol, max_iter, true_every, flexible);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
__global__ void solve_record_kernel(SolveRecord* rec, PcgState* st, int flexible, int stage, int captured) {
    const double rr = st->true_checks ? st->rr_true : st->rr;
    const double rel = st->bb > 0.0 ? sqrt(rr / st->bb) : 0.0;
    const int conv = st->done == 1;
    rec->iters_total += (unsigned long long)st->iter;
    if (stage == 0) {
        rec->iters = st->iter;
        rec->plain_iters = 0;
        rec->fell_back = flexible && !conv;
        rec->solves += 1;
        rec->fallbacks += (unsigned long long)(flexible && !conv);
        if (captured) {
            if (flexible) rec->chunks_primary += (unsigned long long)st->chunks;
            else rec->chunks_plain += (unsigned long long)st->chunks;
            rec->fallbacks_captured += (unsigned long long)(flexible && !conv);
        }
    } else {
        rec->plain_iters = st->iter;
        if (captured) rec->chunks_plain += (unsigned long long)st->chunks;
    }
    rec->converged = conv;
    rec->rel_residual = rel;
    rec->warm_ok = conv;
}
int nat_launch_solve_record(SolveRecord* rec, PcgState* st, int flexible, int stage, int captured, cudaStream_t s) {
    solve_record_kernel<<<1, 1, 0, s>>>(rec, st, flexible, stage, captured);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
__global__ void cond_set_kernel(cudaGraphConditionalHandle h, unsigned int v) { cudaGraphSetConditional(h, v); }
int nat_launch_cond_set(cudaGraphConditionalHandle h, unsigned int v, cudaStream_t s) {
    cond_set_kernel<<<1, 1, 0, s>>>(h, v);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
__global__ void fallback_cond_kernel(cudaGraphConditionalHandle h, const PcgState* st) {
    cudaGraphSetConditional(h, st->done != 1 ? 1u : 0u);
}
int nat_launch_fallback_cond(cudaGraphConditionalHandle h, const PcgState* st, cudaStream_t s) {
    fallback_cond_kernel<<<1, 1, 0, s>>>(h, st);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
// the rules of the host loop of flip_solve_frame, on the device: sub-steps
// of min(max_dt, 0.7 h / max |v component|, the rest of the frame); a
// collapsed dt or 100,000 sub-steps stop the frame with fs->error set
__global__ void frame_ctl_kernel(cudaGraphConditionalHandle h, FrameState* fs, const uint32_t* vmax_bits, float gravity_y) {
    const float vmax = __uint_as_float(*vmax_bits);
    double dt = fmin(fs->max_dt, fs->frame_dt - fs->t);
    if (vmax > 0.0f) dt = fmin(dt, 0.7 * fs->h / (double)vmax);
    if (!(dt > 1e-9 * fs->frame_dt) || fs->substeps >= 100000) {
        fs->error = 1;
        dt = 0.0;
    }
    fs->t += dt;
    fs->dt = (float)dt;
    fs->gdt = (float)((double)gravity_y * dt);
    fs->substeps += 1;
    cudaGraphSetConditional(h, (!fs->error && fs->frame_dt - fs->t > 1e-12 * fs->frame_dt) ? 1u : 0u);
}
int nat_launch_frame_ctl(cudaGraphConditionalHandle h, FrameState* fs, const uint32_t* vmax_bits, float gravity_y,
                         cudaStream_t s) {
    frame_ctl_kernel<<<1, 1, 0, s>>>(h, fs, vmax_bits, gravity_y);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
__global__ void frame_init_kernel(FrameState* fs, double frame_dt, double max_dt, double h) {
    FrameState f{};
    f.frame_dt = frame_dt;
    f.max_dt = max_dt;
    f.h = h;
    *fs = f;
}
int nat_launch_frame_init(FrameState* fs, double frame_dt, double max_dt, double h, cudaStream_t s) {
    frame_init_kernel<<<1, 1, 0, s>>>(fs, frame_dt, max_dt, h);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
__global__ void step_dt_kernel(FrameState* fs, double dt, float gravity_y) {
    fs->dt = (float)dt;
    fs->gdt = (float)((double)gravity_y * dt);
}
int nat_launch_step_dt(FrameState* fs, double dt, float gravity_y, cudaStream_t s) {
    step_dt_kernel<<<1, 1, 0, s>>>(fs, dt, gravity_y);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

// largest |velocity component| over the particles, as the bits of a
// non-negative float (their unsigned order is the float order); *out must be 0
__global__ void __launch_bounds__(256) nat_vmax_kernel(uint64_t n, const float* __restrict__ vx,
                                                       const float* __restrict__ vy, const float* __restrict__ vz,
                                                       uint32_t* __restrict__ out) {
    float m = 0.0f;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        m = fmaxf(m, fmaxf(fabsf(vx[i]), fmaxf(fabsf(vy[i]), fabsf(vz[i]))));
    uint32_t b = __float_as_uint(m);
    b = __reduce_max_sync(0xFFFFFFFFu, b);
    if ((threadIdx.x & 31) == 0 && b) atomicMax(out, b);
}
int nat_launch_vmax(uint64_t n, const float* const* V, uint32_t* d_out, int grid, cudaStream_t s) {
    FLIP_CUDA_TRY(cudaMemsetAsync(d_out, 0, sizeof(uint32_t), s));
    nat_vmax_kernel<<<grid, 256, 0, s>>>(n, V[0], V[1], V[2], d_out);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_project(const uint32_t* tiles, const uint32_t* d_count, const NatDims& D, const double* phi,
                       const float* phig, const uint8_t* type, float* const* U, int grid, cudaStream_t s,
                       float* const* lin) {
    float* const nl[3] = {nullptr, nullptr, nullptr};
    float* const* L = lin ? lin : nl;
    nat_project_kernel<<<grid, 512, 0, s>>>(tiles, d_count, D, phi, phig, type, U[0], U[1], U[2], L[0], L[1], L[2]);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int nat_launch_g2p(const NatG2PMaps& M, const uint32_t* tile_keys, const uint32_t* starts, const uint32_t* d_ntiles,
                   uint64_t n, const NatDims& D, float dt, float flip, const float* const* U, const float* const* O,
                   const float* const* P, const float* const* V, float* const* Pout, float* const* Vout,
                   uint32_t* keys_out, const uint8_t* solid_type, float3 usolid, const float* dt_p, uint32_t* err,
                   int grid, cudaStream_t s) {
    static bool attr_done = false;
    if (!attr_done) {
        FLIP_CUDA_TRY(cudaFuncSetAttribute(nat_g2p_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kG2PSmem));
        attr_done = true;
    }
    if (n)
        nat_g2p_tile_kernel<<<grid, kG2PThreads, kG2PSmem, s>>>(M.u[0], M.u[1], M.u[2], M.o[0], M.o[1], M.o[2], tile_keys,
                                                               starts, d_ntiles, n, D, dt, flip, U[0], U[1], U[2], O[0],
                                                               O[1], O[2], P[0], P[1], P[2], V[0], V[1], V[2], Pout[0],
                                                               Pout[1], Pout[2], Vout[0], Vout[1], Vout[2], keys_out,
                                                               solid_type, usolid, dt_p, err);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

// ------------------------------------------------------- tensor maps
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static std::mutex mu;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!fn) {
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
    }
    return fn;
}

int encode_tensor_map(CUtensorMap* map, CUtensorMapDataType dtype, int rank, const void* base, const uint64_t* dims,
                      const uint64_t* strides_bytes, const uint32_t* box) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = tensor_map_encoder();
    if (!fn) {
        set_error_text("cuTensorMapEncodeTiled is not available from the driver");
        return FLIP_ERR_CUDA;
    }
    if (reinterpret_cast<uintptr_t>(base) & 255) {
        set_error_text("tensor map: base not 256-byte aligned");
        return FLIP_ERR_ARG;
    }
    cuuint64_t d[5];
    cuuint64_t st[4];
    cuuint32_t b[5], es[5];
    for (int i = 0; i < rank; ++i) {
        d[i] = dims[i];
        b[i] = box[i];
        es[i] = 1;
        if (i + 1 < rank) {
            st[i] = strides_bytes[i];
            if (st[i] % 16) {
                set_error_text("tensor map: stride not a multiple of 16 bytes");
                return FLIP_ERR_ARG;
            }
        }
    }
    CUresult r = fn(map, dtype, (cuuint32_t)rank, const_cast<void*>(base), d, st, b, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error_text("cuTensorMapEncodeTiled failed");
        return FLIP_ERR_CUDA;
    }
    return FLIP_OK;
}

int encode_grid_map_f32(CUtensorMap* map, const float* base, int nx, int ny, int nz, int bx, int by, int bz) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = tensor_map_encoder();
    if (!fn) {
        set_error_text("cuTensorMapEncodeTiled is not available from the driver");
        return FLIP_ERR_CUDA;
    }
    if ((bx * 4) % 16 || (nx * 4) % 16 || (reinterpret_cast<uintptr_t>(base) & 255)) {
        set_error_text("tensor map: box or row not a multiple of 16 bytes, or base not 256-byte aligned");
        return FLIP_ERR_ARG;
    }
    const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
    const cuuint64_t strides[2] = {(cuuint64_t)nx * 4, (cuuint64_t)nx * ny * 4};
    const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz};
    const cuuint32_t es[3] = {1, 1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error_text("cuTensorMapEncodeTiled failed");
        return FLIP_ERR_CUDA;
    }
    return FLIP_OK;
}

int nat_make_g2p_maps(NatG2PMaps& M, float* const* ulin, float* const* olin, const NatDims& D) {
    for (int c = 0; c < 3; ++c) {
        if (int rc = encode_grid_map_f32(&M.u[c], ulin[c], D.nx, D.ny, D.nz, kGBx, kGBy, kGBz)) return rc;
        if (int rc = encode_grid_map_f32(&M.o[c], olin[c], D.nx, D.ny, D.nz, kGBx, kGBy, kGBz)) return rc;
    }
    return FLIP_OK;
}

}  // namespace flip
