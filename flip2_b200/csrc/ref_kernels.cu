// ref_kernels.cu -- the reference engine's math on sm_100a, FP64 as in the
// reference (all particle and voxel state is CudaVec<double>).
//
// Each kernel restates one reference kernel with the same arithmetic so that
// integer outputs are bit-exact and floating-point outputs agree to rounding.
// What changes is the execution shape: one CTA of 128 threads per occupied
// root cell instead of 32, the three axes of P2G/G2P/divergence/projection in
// one launch instead of three, the voxel-activation predicate evaluated once
// (its 512-bit mask is kept for the compaction) instead of twice, and the
// tile-local red-black SOR iterated in shared memory for a whole convergence
// check interval instead of two launches per iteration.
//
// The reference's behaviours that change results are kept:
//   - the activation solid test takes the tile origin from the key of
//     particle blockIdx.x (not the node's first particle) and computes the
//     voxel's y index as (i % 8 * 8) / 8, which equals its x index
//     (particles.cu:99,118);
//   - the z-apron copy of the divergence indexes x with the z coordinate
//     (voxelSolveFunctions.cu:85);
//   - the y-row table stores root-cell ids that are later compared with node
//     counts (particleToGridFunctions.cu:369, voxelSolveFunctions.cu:138-156);
//   - G2P skips voxels whose velocity is exactly zero (particles.cu:649).
#include "common.cuh"
#include "ref_kernels.cuh"
#include <curand_kernel.h>

namespace flip {

__device__ __forceinline__ uint32_t sat_u32_d(double v) {
    return (uint32_t)__double2uint_rz(v);  // saturating: negative/NaN -> 0
}
__device__ __forceinline__ uint32_t sat_u32_f(float v) { return (uint32_t)__float2uint_rz(v); }

__device__ __forceinline__ double ref_dist(double dx, double dy, double dz) {
    return sqrt(fma(dx, dx, fma(dy, dy, dz * dz)));
}
__device__ __forceinline__ double ref_scw(const flip_grid& g) { return (double)(g.cellSize / 4.0f); }
__device__ __forceinline__ double ref_local(double p, float neg, uint32_t gid, float cell, double scw) {
    double t = p - (double)neg;
    float prod = __fmul_rn((float)gid, cell);
    t = t - (double)prod;
    return t + 2.0 * scw;
}
__device__ __forceinline__ void ref_decompose(uint32_t key, const flip_grid& g, uint32_t& gx, uint32_t& gy, uint32_t& gz) {
    uint32_t xy = g.sizeX * g.sizeY;
    uint32_t m = key % xy;
    gz = key / xy;
    gy = m / g.sizeX;
    gx = m % g.sizeX;
}

// ----------------------------------------------------------------- keys
// rootCell (particleToGridFunctions.cu:19-45)
__global__ void ref_keys_kernel(double* __restrict__ px, double* __restrict__ py, double* __restrict__ pz, uint64_t n,
                                flip_grid g, uint32_t* __restrict__ keys, uint32_t* __restrict__ idx) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float ux = fmaf((float)g.sizeX, g.cellSize, g.negX);
    const float uy = fmaf((float)g.sizeY, g.cellSize, g.negY);
    const float uz = fmaf((float)g.sizeZ, g.cellSize, g.negZ);
    double x = px[i], y = py[i], z = pz[i];
    if (x < (double)g.negX) { x = g.negX; px[i] = x; } else if (x > (double)ux) { x = ux; px[i] = x; }
    if (y < (double)g.negY) { y = g.negY; py[i] = y; } else if (y > (double)uy) { y = uy; py[i] = y; }
    if (z < (double)g.negZ) { z = g.negZ; pz[i] = z; } else if (z > (double)uz) { z = uz; pz[i] = z; }
    uint32_t kx = sat_u32_f(floorf(__double2float_rn(__ddiv_rn(x - (double)g.negX, (double)g.cellSize))));
    uint32_t ky = sat_u32_f(floorf(__double2float_rn(__ddiv_rn(y - (double)g.negY, (double)g.cellSize))));
    uint32_t kz = sat_u32_f(floorf(__double2float_rn(__ddiv_rn(z - (double)g.negZ, (double)g.cellSize))));
    keys[i] = kx + ky * g.sizeX + kz * g.sizeX * g.sizeY;
    if (idx) idx[i] = (uint32_t)i;
}

// ------------------------------------------------------------ y-row table
__global__ void ref_ydim_fill_kernel(uint32_t* table, uint32_t rows, uint32_t nodes) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < rows) table[i] = nodes;
}
// getYDimPositionFirstInRow (particleToGridFunctions.cu:355-372)
__global__ void ref_ydim_rows_kernel(const uint32_t* __restrict__ starts, const uint32_t* __restrict__ keys, uint32_t nodes,
                                     flip_grid g, uint32_t* __restrict__ table) {
    uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nodes) return;
    uint32_t prev = idx ? keys[starts[idx - 1]] : nodes;
    uint32_t cur = keys[starts[idx]];
    uint32_t pr = prev / g.sizeX, cr = cur / g.sizeX;
    if (pr != cr && cr < g.sizeY * g.sizeZ) table[cr] = cur;
}

// ------------------------------------------------------- voxel activation
constexpr int kNodeThreads = 128;

// solid test of local voxel i of the tile whose origin comes from particle
// b's key (particles.cu:97-130, 203-247), y index computed as written (Q3)
__device__ __forceinline__ bool ref_tile_solid(uint32_t i, uint32_t gx, uint32_t gy, uint32_t gz, const flip_grid& g) {
    uint32_t vx = i % 8u, vy = (i % 8u * 8u) / 8u, vz = i / 64u;
    uint32_t gvx = gx * 8u + vx, gvy = gy * 8u + vy, gvz = gz * 8u + vz;
    const double fr = 2.0;
    if ((double)gvx < fr || (double)gvy < fr || (double)gvz < fr) return true;
    if ((double)gvx > (double)(g.sizeX * 8u) + fr || (double)gvy > (double)(g.sizeY * 8u) + fr ||
        (double)gvz > (double)(g.sizeZ * 8u) + fr)
        return true;
    return false;
}

// true when ref_tile_solid is false for every voxel of the tile: its voxel
// coordinates run over gx*8 .. gx*8+7 in x and y (the y index is the x index)
// and gz*8 .. gz*8+7 in z, and the test is monotone in each, so the tile's
// corners decide (tiles away from the domain faces, nearly all of them)
__device__ __forceinline__ bool ref_tile_clear(uint32_t gx, uint32_t gy, uint32_t gz, const flip_grid& g) {
    const double fr = 2.0;
    if ((double)(gx * 8u) < fr || (double)(gy * 8u) < fr || (double)(gz * 8u) < fr) return false;
    if ((double)(gx * 8u + 7u) > (double)(g.sizeX * 8u) + fr || (double)(gy * 8u + 7u) > (double)(g.sizeY * 8u) + fr ||
        (double)(gz * 8u + 7u) > (double)(g.sizeZ * 8u) + fr)
        return false;
    return true;
}

// ref_dist(dx, dy, dz) < R without the square root where the sum of squares
// s decides it: the square root is correctly rounded and monotone, so it
// comes out below R exactly when s lies below the square of the midpoint
// between R and the double below R, which is within a relative 2^-52 of R^2.
// s below lo = R^2 (1 - 2^-48) is inside, s at or above hi = R^2 (1 + 2^-48)
// is outside (both bounds hold with the roundings of R^2 and of the
// products); in the band between, the square root decides, as in ref_dist.
__device__ __forceinline__ bool ref_within(double dx, double dy, double dz, double R, double lo, double hi) {
    const double s = fma(dx, dx, fma(dy, dy, dz * dz));
    if (s < lo) return true;
    if (s >= hi) return false;
    return sqrt(s) < R;
}

struct RefLocal {
    double lx, ly, lz;
    uint32_t sx, sy, sz;
};
__device__ __forceinline__ RefLocal ref_particle_local(const double* px, const double* py, const double* pz,
                                                      const uint32_t* keys, uint32_t idx, const flip_grid& g, double scw) {
    uint32_t qx, qy, qz;
    ref_decompose(keys[idx], g, qx, qy, qz);
    RefLocal r;
    r.lx = ref_local(px[idx], g.negX, qx, g.cellSize, scw);
    r.ly = ref_local(py[idx], g.negY, qy, g.cellSize, scw);
    r.lz = ref_local(pz[idx], g.negZ, qz, g.cellSize, scw);
    r.sx = sat_u32_d(floor(r.lx / scw));
    r.sy = sat_u32_d(floor(r.ly / scw));
    r.sz = sat_u32_d(floor(r.lz / scw));
    return r;
}

// getNumberVoxelsUsedPerNode (particles.cu:88-190): mask + count per node.
// A warp per node (kVoxWarps nodes per CTA): the 512 solid tests as 16
// ballots (none for a tile away from the domain faces, whose tests all
// fail), then the node's particles in order, the 64 points of a particle's
// 4 x 4 x 4 stencil spread over the lanes (two each); a lane loads and
// prepares one particle of each round of 32, so the loads overlap.  The tests
// and their arithmetic are the reference's; only the work is spread.  Its
// loops run x from sx - 2 while (unsigned) x < sx + 2, so a stencil
// coordinate below 2 on any axis leaves a particle without marks, and points
// outside the 8^3 tile never mark: both are tested before the distances.
constexpr int kVoxWarps = 8;
__global__ void __launch_bounds__(32 * kVoxWarps) ref_voxel_counts_kernel(
    const uint32_t* __restrict__ starts, const uint32_t* __restrict__ keys, uint32_t nodes, uint64_t n,
    const double* __restrict__ px, const double* __restrict__ py, const double* __restrict__ pz, flip_grid g,
    uint32_t* __restrict__ counts, uint32_t* __restrict__ masks) {
    __shared__ uint32_t mark[kVoxWarps][16];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t b = blockIdx.x * kVoxWarps + (uint32_t)w;
    if (b >= nodes) return;  // a whole warp; nothing below synchronises the CTA
    uint32_t* M = mark[w];
    // the node's particle range, loaded with the key below
    const uint32_t first = starts[b], last = (b == nodes - 1) ? (uint32_t)n : starts[b + 1];
    uint32_t gx, gy, gz;
    ref_decompose(keys[b], g, gx, gy, gz);  // Q3: particle b's key, not the node's
    if (ref_tile_clear(gx, gy, gz, g)) {
        if (lane < 16) M[lane] = 0u;
    } else {
#pragma unroll 4
        for (int q = 0; q < 16; ++q) {
            const uint32_t bits = __ballot_sync(0xffffffffu, ref_tile_solid((uint32_t)(q * 32 + lane), gx, gy, gz, g));
            if (lane == 0) M[q] = bits;
        }
    }
    __syncwarp();
    const double scw = ref_scw(g), hs = scw / 2.0, R = 2.0 * scw;
    const double R2 = R * R, lo = R2 * (1.0 - 0x1p-48), hi = R2 * (1.0 + 0x1p-48);
    // up to 32 of the node's particles at a time: lane j loads particle j and
    // works out its local coordinates (the loads and divisions of all of
    // them in one round), then the warp walks them in order, each lane
    // taking two of the 64 points of the particle's stencil
    for (uint32_t i0 = first; i0 < last; i0 += 32u) {
        RefLocal Lj{};
        bool ok = false;
        if (i0 + (uint32_t)lane < last) {
            Lj = ref_particle_local(px, py, pz, keys, i0 + (uint32_t)lane, g, scw);
            ok = !(Lj.sx < 2u || Lj.sy < 2u || Lj.sz < 2u);
        }
        for (uint32_t live = __ballot_sync(0xffffffffu, ok); live; live &= live - 1u) {
            const int j = __ffs(live) - 1;
            RefLocal L;
            L.lx = __shfl_sync(0xffffffffu, Lj.lx, j);
            L.ly = __shfl_sync(0xffffffffu, Lj.ly, j);
            L.lz = __shfl_sync(0xffffffffu, Lj.lz, j);
            L.sx = __shfl_sync(0xffffffffu, Lj.sx, j);
            L.sy = __shfl_sync(0xffffffffu, Lj.sy, j);
            L.sz = __shfl_sync(0xffffffffu, Lj.sz, j);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int pt = lane + 32 * h;
                const int x = (int)(L.sx - 2u) + (pt >> 4), y = (int)(L.sy - 2u) + ((pt >> 2) & 3),
                          z = (int)(L.sz - 2u) + (pt & 3);
                if ((uint32_t)x >= 8u || (uint32_t)y >= 8u || (uint32_t)z >= 8u) continue;
                const double dx = L.lx - x * scw, dy = L.ly - y * scw, dz = L.lz - z * scw;
                if (ref_within(dx, dy + hs, dz + hs, R, lo, hi) || ref_within(dx + hs, dy, dz + hs, R, lo, hi) ||
                    ref_within(dx + hs, dy + hs, dz, R, lo, hi)) {
                    const int v = x + y * 8 + z * 64;
                    atomicOr(&M[v >> 5], 1u << (v & 31));
                }
            }
        }
    }
    __syncwarp();
    const uint32_t bits = lane < 16 ? M[lane] : 0u;
    if (lane < 16) masks[(size_t)b * 16 + lane] = bits;
    uint32_t c = __popc(bits);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) counts[b] = c;
}

// generateVoxelIDs (particles.cu:192-321): compaction from the mask, a warp
// per node; lane l writes bit l of each mask word
__global__ void __launch_bounds__(32 * kVoxWarps) ref_voxel_ids_kernel(
    const uint32_t* __restrict__ keys, uint32_t nodes, const uint32_t* __restrict__ masks,
    const uint32_t* __restrict__ node_voxels, flip_grid g, uint32_t* __restrict__ voxel_ids, int8_t* __restrict__ solids) {
    const int lane = threadIdx.x & 31;
    const uint32_t b = blockIdx.x * kVoxWarps + (threadIdx.x >> 5);
    if (b >= nodes) return;
    const uint32_t m = lane < 16 ? masks[(size_t)b * 16 + lane] : 0u;
    // exclusive prefix of the words' popcounts over lanes 0..15
    uint32_t inc = __popc(m);
#pragma unroll
    for (int o = 1; o < 16; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    const uint32_t pre = inc - __popc(m);
    uint32_t gx, gy, gz;
    ref_decompose(keys[b], g, gx, gy, gz);
    const uint32_t start = b ? node_voxels[b - 1] : 0u;
    const uint32_t below = (1u << lane) - 1u;
    const bool clear = ref_tile_clear(gx, gy, gz, g);
    // the mask words that hold a voxel, in order
    for (uint32_t rest = __ballot_sync(0xffffffffu, m != 0u); rest; rest &= rest - 1u) {
        const int q = __ffs(rest) - 1;
        const uint32_t word = __shfl_sync(0xffffffffu, m, q), base = __shfl_sync(0xffffffffu, pre, q);
        if ((word >> lane) & 1u) {
            const uint32_t i = (uint32_t)(q * 32 + lane);
            const uint32_t pos = start + base + __popc(word & below);
            voxel_ids[pos] = i;
            solids[pos] = (!clear && ref_tile_solid(i, gx, gy, gz, g)) ? 1 : 0;
        }
    }
}

// ------------------------------------------------------------- P2G / G2P
__device__ __forceinline__ void ref_face_base(int dim, double hs, double& bx, double& by, double& bz) {
    if (dim == 0) { by += hs; bz += hs; }
    else if (dim == 1) { bx += hs; bz += hs; }
    else { by += hs; bx += hs; }
}
__device__ __forceinline__ double ref_weight(double d, double R) { return (d > R) ? 0.0 : 1.0 - d / R; }

// gatherParticleVelsToVoxels for X, Y and Z in one launch (particles.cu:379-488)
__global__ void __launch_bounds__(kNodeThreads) ref_p2g_kernel(
    const uint32_t* __restrict__ starts, const uint32_t* __restrict__ keys, uint32_t nodes, uint64_t n,
    const double* __restrict__ px, const double* __restrict__ py, const double* __restrict__ pz,
    const double* __restrict__ vx, const double* __restrict__ vy, const double* __restrict__ vz,
    const uint32_t* __restrict__ node_voxels, const uint32_t* __restrict__ voxel_ids, const int8_t* __restrict__ solids,
    flip_grid g, double* __restrict__ ux, double* __restrict__ uy, double* __restrict__ uz) {
    __shared__ double U[3][512];
    __shared__ double W[3][512];
    __shared__ int8_t S[512];
    const uint32_t b = blockIdx.x;
    for (int i = threadIdx.x; i < 512; i += kNodeThreads) {
        U[0][i] = U[1][i] = U[2][i] = 0.0;
        W[0][i] = W[1][i] = W[2][i] = 0.0;
        S[i] = 0;
    }
    __syncthreads();
    const uint32_t vs = b ? node_voxels[b - 1] : 0u, ve = node_voxels[b];
    for (uint32_t k = vs + threadIdx.x; k < ve; k += kNodeThreads) S[voxel_ids[k]] = solids[k];
    const uint32_t last = (b == nodes - 1) ? (uint32_t)n : starts[b + 1];
    const double scw = ref_scw(g), hs = scw / 2.0, R = 2.0 * scw;
    for (uint32_t idx = starts[b] + threadIdx.x; idx < last; idx += kNodeThreads) {
        RefLocal L = ref_particle_local(px, py, pz, keys, idx, g, scw);
        const double v[3] = {vx[idx], vy[idx], vz[idx]};
        for (int x = (int)(L.sx - 2u); (uint32_t)x < L.sx + 2u; ++x)
            for (int y = (int)(L.sy - 2u); (uint32_t)y < L.sy + 2u; ++y)
                for (int z = (int)(L.sz - 2u); (uint32_t)z < L.sz + 2u; ++z) {
                    if (!((uint32_t)x < 8u && (uint32_t)y < 8u && (uint32_t)z < 8u)) continue;
                    const int id = x + y * 8 + z * 64;
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        double bx = x * scw, by = y * scw, bz = z * scw;
                        ref_face_base(d, hs, bx, by, bz);
                        double w = ref_weight(ref_dist(L.lx - bx, L.ly - by, L.lz - bz), R);
                        atomicAdd(&W[d][id], w);
                        atomicAdd(&U[d][id], __dmul_rn(w, v[d]));
                    }
                }
    }
    __syncthreads();
    for (uint32_t k = vs + threadIdx.x; k < ve; k += kNodeThreads) {
        uint32_t id = voxel_ids[k];
        bool sol = S[id] != 0;
        ux[k] = (sol ? 0.0 : U[0][id]) / (W[0][id] + 0.0000001);
        uy[k] = (sol ? 0.0 : U[1][id]) / (W[1][id] + 0.0000001);
        uz[k] = (sol ? 0.0 : U[2][id]) / (W[2][id] + 0.0000001);
    }
}

// gatherVoxelVelsToParticles for X, Y and Z (particles.cu:562-662)
__global__ void __launch_bounds__(kNodeThreads) ref_g2p_kernel(
    const uint32_t* __restrict__ starts, const uint32_t* __restrict__ keys, uint32_t nodes, uint64_t n,
    const double* __restrict__ px, const double* __restrict__ py, const double* __restrict__ pz,
    const uint32_t* __restrict__ node_voxels, const uint32_t* __restrict__ voxel_ids,
    const double* __restrict__ ux, const double* __restrict__ uy, const double* __restrict__ uz, flip_grid g,
    double* __restrict__ vx, double* __restrict__ vy, double* __restrict__ vz) {
    __shared__ double U[3][512];
    const uint32_t b = blockIdx.x;
    for (int i = threadIdx.x; i < 512; i += kNodeThreads) U[0][i] = U[1][i] = U[2][i] = 0.0;
    __syncthreads();
    const uint32_t vs = b ? node_voxels[b - 1] : 0u, ve = node_voxels[b];
    for (uint32_t k = vs + threadIdx.x; k < ve; k += kNodeThreads) {
        uint32_t id = voxel_ids[k];
        U[0][id] = ux[k];
        U[1][id] = uy[k];
        U[2][id] = uz[k];
    }
    __syncthreads();
    const uint32_t last = (b == nodes - 1) ? (uint32_t)n : starts[b + 1];
    const double scw = ref_scw(g), hs = scw / 2.0, R = 2.0 * scw;
    for (uint32_t idx = starts[b] + threadIdx.x; idx < last; idx += kNodeThreads) {
        RefLocal L = ref_particle_local(px, py, pz, keys, idx, g, scw);
        double vel[3] = {0.0, 0.0, 0.0}, ws[3] = {0.0, 0.0, 0.0};
        for (int x = (int)(L.sx - 2u); (uint32_t)x < 8u && (uint32_t)x < L.sx + 2u; ++x)
            for (int y = (int)(L.sy - 2u); (uint32_t)y < 8u && (uint32_t)y < L.sy + 2u; ++y)
                for (int z = (int)(L.sz - 2u); (uint32_t)z < 8u && (uint32_t)z < L.sz + 2u; ++z) {
                    const int id = x + y * 8 + z * 64;
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        double bx = x * scw, by = y * scw, bz = z * scw;
                        ref_face_base(d, hs, bx, by, bz);
                        double w = ref_weight(ref_dist(L.lx - bx, L.ly - by, L.lz - bz), R);
                        double u = U[d][id];
                        if (u != 0.0) {  // Q10
                            ws[d] += w;
                            vel[d] = fma(w, u, vel[d]);
                        }
                    }
                }
        vx[idx] = vel[0] / (ws[0] + 0.00000001);
        vy[idx] = vel[1] / (ws[1] + 0.00000001);
        vz[idx] = vel[2] / (ws[2] + 0.00000001);
    }
}

// advectParticlePositions for the three axes (particles.cu:664-669)
__global__ void ref_advect_kernel(uint64_t n, double dt, double* __restrict__ px, double* __restrict__ py,
                                  double* __restrict__ pz, const double* __restrict__ vx, const double* __restrict__ vy,
                                  const double* __restrict__ vz) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    px[i] = fma(dt, vx[i], px[i]);
    py[i] = fma(dt, vy[i], py[i]);
    pz[i] = fma(dt, vz[i], pz[i]);
}

// --------------------------------------------------------------- pressure
// applyGravityKernel / removeGravityKernel (voxelSolveFunctions.cu:160-175)
__global__ void ref_gravity_kernel(uint64_t nvox, const int8_t* __restrict__ solids, double* __restrict__ uy, double dt,
                                   int remove) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nvox || solids[i]) return;
    const double c = (double)(-9.8f);
    uy[i] = remove ? fma(-c, dt, uy[i]) : fma(c, dt, uy[i]);
}

__device__ void ref_apron_add(uint32_t nid, const uint32_t* node_voxels, const uint32_t* voxel_ids, const double* data,
                              double* S, int xo, int yo, int zo) {
    const uint32_t vs = nid ? node_voxels[nid - 1] : 0u, ve = node_voxels[nid];
    for (uint32_t k = vs + threadIdx.x; k < ve; k += blockDim.x) {
        uint32_t id = voxel_ids[k];
        uint32_t sx = id % 8u, sy = (id % 64u) / 8u, sz = id / 64u;
        uint32_t tx = sx, ty = sy, tz = sz;
        int t = -1;
        if (xo < 0) { if (sx >= 8u + (uint32_t)xo) { tx = sx - 8u - (uint32_t)xo; t = tx + ty * 8 + tz * 64; } }
        else if (xo > 0) { if (sx < (uint32_t)xo) { tx = 8u - (uint32_t)xo + sx; t = tx + ty * 8 + tz * 64; } }
        else if (yo < 0) { if (sy >= 8u + (uint32_t)yo) { ty = sy - 8u - (uint32_t)yo; t = tx + ty * 8 + tz * 64; } }
        else if (yo > 0) { if (sy < (uint32_t)yo) { ty = 8u - (uint32_t)yo + sy; t = tx + ty * 8 + tz * 64; } }
        else if (zo < 0) { if (sz >= 8u + (uint32_t)zo) { tz = sz - 8u - (uint32_t)zo; t = tz + ty * 8 + tz * 64; } }  // Q6
        else if (zo > 0) { if (sz < (uint32_t)zo) { tz = 8u - (uint32_t)zo + sz; t = tx + ty * 8 + tz * 64; } }
        if (t >= 0) atomicAdd(&S[t], data[k]);
    }
}

// cudaCalcDivU for X, Y and Z (voxelSolveFunctions.cu:97-271): apron
// contributions of the x/y/z neighbours, then forward differences
__global__ void __launch_bounds__(kNodeThreads) ref_divergence_kernel(
    uint32_t nodes, const uint32_t* __restrict__ node_voxels, const uint32_t* __restrict__ voxel_ids,
    const double* __restrict__ ux, const double* __restrict__ uy, const double* __restrict__ uz, flip_grid g,
    const uint32_t* __restrict__ ytable, const uint32_t* __restrict__ starts, const uint32_t* __restrict__ keys,
    double* __restrict__ divU) {
    __shared__ double S[3][512];
    const uint32_t b = blockIdx.x;
    for (int i = threadIdx.x; i < 512; i += kNodeThreads) S[0][i] = S[1][i] = S[2][i] = 0.0;
    __syncthreads();
    const double* data[3] = {ux, uy, uz};
    const uint32_t vs = b ? node_voxels[b - 1] : 0u, ve = node_voxels[b];
    for (uint32_t k = vs + threadIdx.x; k < ve; k += kNodeThreads) {
        uint32_t id = voxel_ids[k];
        S[0][id] = ux[k];
        S[1][id] = uy[k];
        S[2][id] = uz[k];
    }
    __syncthreads();
    const uint32_t cur = keys[starts[b]];
    const uint32_t cx = cur % g.sizeX, cy = (cur % (g.sizeX * g.sizeY)) / g.sizeX, cz = cur / (g.sizeX * g.sizeY);
    const int xl = (int)(cx - 1u), xr = (int)(cx + 1u), yl = (int)(cy - 1u), yr = (int)(cy + 1u), zl = (int)(cz - 1u),
              zr = (int)(cz + 1u);
    const int T = 4;
    // y-row table lookups; a key on the upper face of the box aliases past the
    // last row (the reference reads out of bounds there), treated as "none"
    const uint32_t rows = g.sizeY * g.sizeZ;
    auto row = [&](uint32_t r) -> uint32_t { return r < rows ? ytable[r] : nodes; };
    const uint32_t nyl = yl >= 0 ? row((uint32_t)yl + cz * g.sizeY) : nodes;
    const uint32_t nyr = (uint32_t)yr < g.sizeY ? row((uint32_t)yr + cz * g.sizeY) : nodes;
    const uint32_t nzl = zl >= 0 ? row((uint32_t)zl * g.sizeY + cy) : nodes;
    const uint32_t nzr = (uint32_t)zr < g.sizeZ ? row((uint32_t)zr * g.sizeY + cy) : nodes;
    const bool hxl = xl >= 0 && b > 0 && keys[starts[b - 1]] == cur - 1u;
    const bool hxr = (uint32_t)xr < g.sizeX && b < nodes - 1 && keys[starts[b + 1]] == cur + 1u;
    for (int d = 0; d < 3; ++d) {
        if (hxl) ref_apron_add(b - 1, node_voxels, voxel_ids, data[d], S[d], -T, 0, 0);
        __syncthreads();
        if (hxr) ref_apron_add(b + 1, node_voxels, voxel_ids, data[d], S[d], T, 0, 0);
        __syncthreads();
        if (nyl < nodes) ref_apron_add(nyl, node_voxels, voxel_ids, data[d], S[d], 0, -T, 0);
        __syncthreads();
        if (nyr < nodes) ref_apron_add(nyr, node_voxels, voxel_ids, data[d], S[d], 0, T, 0);
        __syncthreads();
        if (nzl < nodes) ref_apron_add(nzl, node_voxels, voxel_ids, data[d], S[d], 0, 0, -T);
        __syncthreads();
        if (nzr < nodes) ref_apron_add(nzr, node_voxels, voxel_ids, data[d], S[d], 0, 0, T);
        __syncthreads();
    }
    for (uint32_t k = vs + threadIdx.x; k < ve; k += kNodeThreads) {
        uint32_t id = voxel_ids[k];
        double dx = (id % 8u < 7u) ? S[0][id + 1] - S[0][id] : 0.0;
        double dy = ((id % 64u) / 8u < 7u) ? S[1][id + 8] - S[1][id] : 0.0;
        double dz = (id / 64u < 7u) ? S[2][id + 64] - S[2][id] : 0.0;
        divU[k] = ((0.0 + dx) + dy) + dz;
    }
}

__device__ __forceinline__ bool ref_is_apron(uint32_t id) {
    uint32_t x = id % 8u, y = (id % 8u * 8u) / 8u, z = id / 64u;  // y as written: equals x
    return x < 1u || x >= 7u || y < 1u || y >= 7u || z < 1u || z >= 7u;
}
__device__ __forceinline__ bool ref_is_red(uint32_t id) {
    uint32_t x = id % 8u, y = (id % 64u) / 8u, z = id / 64u;
    return !((x + y + z) & 1u);
}

// `iters` red+black iterations of GSiteration (voxelSolveFunctions.cu:293-389)
// kept in shared memory: the reference's sweeps never read another node's
// voxels, so iterating in place is the same arithmetic as 2*iters launches.
__global__ void __launch_bounds__(kNodeThreads) ref_gs_kernel(
    uint32_t nodes, const uint32_t* __restrict__ node_voxels, const uint32_t* __restrict__ voxel_ids,
    const int8_t* __restrict__ solids, const double* __restrict__ divU, double* __restrict__ p, double* __restrict__ res,
    double scale, double w, uint32_t iters) {
    __shared__ double D[512], P[512], Rr[512];
    __shared__ int8_t S[512];
    __shared__ uint16_t ids[512];
    const uint32_t b = blockIdx.x;
    for (int i = threadIdx.x; i < 512; i += kNodeThreads) { D[i] = 0.0; P[i] = 0.0; Rr[i] = 0.0; S[i] = 0; }
    __syncthreads();
    const uint32_t vs = b ? node_voxels[b - 1] : 0u, ve = node_voxels[b];
    const uint32_t cnt = ve - vs;
    for (uint32_t k = threadIdx.x; k < cnt; k += kNodeThreads) {
        uint32_t id = voxel_ids[vs + k];
        ids[k] = (uint16_t)id;
        D[id] = divU[vs + k];
        P[id] = p[vs + k];
        S[id] = solids[vs + k];
    }
    __syncthreads();
    for (uint32_t it = 0; it < iters; ++it) {
        for (int color = 1; color >= 0; --color) {
            for (uint32_t k = threadIdx.x; k < cnt; k += kNodeThreads) {
                uint32_t v = ids[k];
                Rr[v] = 0.0;  // the pass writes residual 0 for voxels it does not update
                if ((color == (int)ref_is_red(v)) && !S[v] && !ref_is_apron(v)) {
                    double Ad = 0.0, Anx = 0.0, Apx = 0.0, Any = 0.0, Apy = 0.0, Anz = 0.0, Apz = 0.0;
                    if (!S[v - 1]) { if (D[v - 1] != 0.0) Anx = -scale; Ad += scale; }
                    if (!S[v + 1]) { if (D[v + 1] != 0.0) Apx = -scale; Ad += scale; }
                    if (!S[v - 8]) { if (D[v - 8] != 0.0) Any = -scale; Ad += scale; }
                    if (!S[v + 8]) { if (D[v + 8] != 0.0) Apy = -scale; Ad += scale; }
                    if (!S[v - 64]) { if (D[v - 64] != 0.0) Anz = -scale; Ad += scale; }
                    if (!S[v + 64]) { if (D[v + 64] != 0.0) Apz = -scale; Ad += scale; }
                    double s = __dmul_rn(Anx, P[v - 1]);
                    s = fma(Apx, P[v + 1], s);
                    s = fma(Any, P[v - 8], s);
                    s = fma(Apy, P[v + 8], s);
                    s = fma(Anz, P[v - 64], s);
                    s = fma(Apz, P[v + 64], s);
                    double Adg = Ad + 0.000000001;
                    double t = __dsub_rn(__ddiv_rn(-D[v] - s, Adg), P[v]);
                    double pn = fma(w, t, P[v]);
                    P[v] = pn;
                    Rr[v] = __dadd_rn(fma(-Adg, pn, -D[v]), s);
                }
            }
            __syncthreads();
        }
    }
    for (uint32_t k = threadIdx.x; k < cnt; k += kNodeThreads) {
        uint32_t id = ids[k];
        p[vs + k] = P[id];
        res[vs + k] = Rr[id];
    }
}

// pressureToAcceleration for X, Y and Z (voxelSolveFunctions.cu:415-479)
__global__ void __launch_bounds__(kNodeThreads) ref_velocity_update_kernel(
    uint32_t nodes, const uint32_t* __restrict__ node_voxels, const uint32_t* __restrict__ voxel_ids,
    const int8_t* __restrict__ solids, const double* __restrict__ p, double* __restrict__ ux, double* __restrict__ uy,
    double* __restrict__ uz, double scale) {
    __shared__ double P[512];
    __shared__ int8_t S[512];
    const uint32_t b = blockIdx.x;
    for (int i = threadIdx.x; i < 512; i += kNodeThreads) { P[i] = 0.0; S[i] = 0; }
    __syncthreads();
    const uint32_t vs = b ? node_voxels[b - 1] : 0u, ve = node_voxels[b];
    for (uint32_t k = vs + threadIdx.x; k < ve; k += kNodeThreads) {
        uint32_t id = voxel_ids[k];
        P[id] = p[k];
        S[id] = solids[k];
    }
    __syncthreads();
    double* U[3] = {ux, uy, uz};
    const uint32_t stride[3] = {1u, 8u, 64u};
    for (uint32_t k = vs + threadIdx.x; k < ve; k += kNodeThreads) {
        uint32_t v = voxel_ids[k];
        if (S[v] || ref_is_apron(v)) continue;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double dp = 0.0;
            if (!S[v - stride[d]]) dp = __dsub_rn(P[v], P[v - stride[d]]);
            U[d][k] = fma(-dp, scale, U[d][k]);
        }
    }
}

// getMaxFromArray (engine/cudaVec.cu:173-203) as the reference computes it:
// each 512-element block yields the pick of its elements 0 and 256.
__global__ void ref_getmax_kernel(uint64_t n, const double* __restrict__ a, double* __restrict__ out, int absolute) {
    uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t nb = n / 512 + 1;
    if (b >= nb) return;
    uint64_t i0 = b * 512, i1 = b * 512 + 256;
    double s0 = (i0 < n) ? a[i0] : 0.0, s1 = (i1 < n) ? a[i1] : 0.0;
    out[b] = absolute ? ((fabs(s0) > fabs(s1)) ? s0 : s1) : ((s0 > s1) ? s0 : s1);
}

// moveSolids (particles.cu:674-740): particles outside their tile or inside
// a solid voxel are re-seeded at a random point of the node's first solid
// voxel (the reference searches for a solid one, Q8), with the reference's
// launch shape (32 threads per node) so that each thread draws from the same
// curand subsequence.  The search is bounded by the node's own voxel list;
// the reference compares against the cumulative count and can read past it.
__global__ void __launch_bounds__(32) ref_move_solids_kernel(
    uint32_t nodes, uint64_t n, const uint32_t* __restrict__ starts, const uint32_t* __restrict__ keys,
    double* __restrict__ px, double* __restrict__ py, double* __restrict__ pz, const uint32_t* __restrict__ node_voxels,
    const uint32_t* __restrict__ voxel_ids, const int8_t* __restrict__ solids, flip_grid g) {
    __shared__ int8_t S[512];
    __shared__ uint32_t proc[512];
    curandState rs;
    curand_init(1291293829ull, threadIdx.x + blockIdx.x * blockDim.x, 0ull, &rs);
    const uint32_t b = blockIdx.x;
    for (int i = threadIdx.x; i < 512; i += 32) { S[i] = 0; proc[i] = 512u; }
    __syncthreads();
    const uint32_t vs = b ? node_voxels[b - 1] : 0u, ve = node_voxels[b];
    for (uint32_t k = vs + threadIdx.x; k < ve; k += 32) { S[voxel_ids[k]] = solids[k]; proc[k - vs] = voxel_ids[k]; }
    __syncthreads();
    const uint32_t cnt = ve - vs;
    const uint32_t last = (b == nodes - 1) ? (uint32_t)n : starts[b + 1];
    const double scw = ref_scw(g);
    for (uint32_t idx = starts[b] + threadIdx.x; idx < last; idx += 32) {
        uint32_t qx, qy, qz;
        ref_decompose(keys[idx], g, qx, qy, qz);
        double lx = ref_local(px[idx], g.negX, qx, g.cellSize, scw);
        double ly = ref_local(py[idx], g.negY, qy, g.cellSize, scw);
        double lz = ref_local(pz[idx], g.negZ, qz, g.cellSize, scw);
        uint32_t sx = sat_u32_d(floor(lx / scw)), sy = sat_u32_d(floor(ly / scw)), sz = sat_u32_d(floor(lz / scw));
        if (sx >= 8u || sy >= 8u || sz >= 8u || S[sx + sy * 8u + sz * 64u]) {
            uint32_t i = 0;
            while (i < cnt && !S[proc[i]]) ++i;
            uint32_t nv = (i < 512u) ? proc[i] : 512u;
            int nx_ = (int)(nv % 8u), ny_ = (int)((nv % 64u) / 8u), nz_ = (int)(nv / 64u);
            double bx = fma((double)(nx_ - 2), scw, (double)fmaf((float)qx, g.cellSize, g.negX));
            double by = fma((double)(ny_ - 2), scw, (double)fmaf((float)qy, g.cellSize, g.negY));
            double bz = fma((double)(nz_ - 2), scw, (double)fmaf((float)qz, g.cellSize, g.negZ));
            px[idx] = fma((double)curand_uniform(&rs), scw, bx);
            py[idx] = fma((double)curand_uniform(&rs), scw, by);
            pz[idx] = fma((double)curand_uniform(&rs), scw, bz);
        }
    }
}

// reorderGridIndices<double> (radixSortKernels.cu:59-68): out[i] = in[perm[i]]
__global__ void ref_gather_f64_kernel(const uint32_t* __restrict__ perm, uint64_t n, const double* __restrict__ in,
                                      double* __restrict__ out) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        uint32_t s = perm[i];
        out[i] = __ldg(in + (s < n ? s : i));  // a valid permutation always has s < n
    }
}

// ------------------------------------------------------------ launchers
static inline unsigned nblk(uint64_t n, int t) { return (unsigned)((n + t - 1) / t); }

int ref_launch_keys(double* px, double* py, double* pz, uint64_t n, const flip_grid& g, uint32_t* keys, uint32_t* idx,
                    cudaStream_t s) {
    if (n) ref_keys_kernel<<<nblk(n, 256), 256, 0, s>>>(px, py, pz, n, g, keys, idx);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int ref_launch_ydim(const uint32_t* starts, const uint32_t* keys, uint32_t nodes, const flip_grid& g, uint32_t* table,
                    cudaStream_t s) {
    uint32_t rows = g.sizeY * g.sizeZ;
    if (rows) ref_ydim_fill_kernel<<<nblk(rows, 256), 256, 0, s>>>(table, rows, nodes);
    if (nodes) ref_ydim_rows_kernel<<<nblk(nodes, 256), 256, 0, s>>>(starts, keys, nodes, g, table);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int ref_launch_voxel_counts(const uint32_t* starts, const uint32_t* keys, uint32_t nodes, uint64_t n, const double* px,
                            const double* py, const double* pz, const flip_grid& g, uint32_t* counts, uint32_t* masks,
                            cudaStream_t s) {
    if (nodes)
        ref_voxel_counts_kernel<<<(nodes + kVoxWarps - 1) / kVoxWarps, 32 * kVoxWarps, 0, s>>>(starts, keys, nodes, n, px, py,
                                                                                            pz, g, counts, masks);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int ref_launch_voxel_ids(const uint32_t* keys, uint32_t nodes, const uint32_t* masks, const uint32_t* node_voxels,
                         const flip_grid& g, uint32_t* voxel_ids, int8_t* solids, cudaStream_t s) {
    if (nodes)
        ref_voxel_ids_kernel<<<(nodes + kVoxWarps - 1) / kVoxWarps, 32 * kVoxWarps, 0, s>>>(keys, nodes, masks, node_voxels, g,
                                                                                          voxel_ids, solids);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int ref_launch_p2g(const uint32_t* starts, const uint32_t* keys, uint32_t nodes, uint64_t n, const double* px,
                   const double* py, const double* pz, const double* vx, const double* vy, const double* vz,
                   const uint32_t* node_voxels, const uint32_t* voxel_ids, const int8_t* solids, const flip_grid& g,
                   double* ux, double* uy, double* uz, cudaStream_t s) {
    if (nodes)
        ref_p2g_kernel<<<nodes, kNodeThreads, 0, s>>>(starts, keys, nodes, n, px, py, pz, vx, vy, vz, node_voxels, voxel_ids,
                                                      solids, g, ux, uy, uz);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int ref_launch_g2p(const uint32_t* starts, const uint32_t* keys, uint32_t nodes, uint64_t n, const double* px,
                   const double* py, const double* pz, const uint32_t* node_voxels, const uint32_t* voxel_ids,
                   const double* ux, const double* uy, const double* uz, const flip_grid& g, double* vx, double* vy,
                   double* vz, cudaStream_t s) {
    if (nodes)
        ref_g2p_kernel<<<nodes, kNodeThreads, 0, s>>>(starts, keys, nodes, n, px, py, pz, node_voxels, voxel_ids, ux, uy, uz,
                                                      g, vx, vy, vz);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int ref_launch_advect(uint64_t n, double dt, double* px, double* py, double* pz, const double* vx, const double* vy,
                      const double* vz, cudaStream_t s) {
    if (n) ref_advect_kernel<<<nblk(n, 256), 256, 0, s>>>(n, dt, px, py, pz, vx, vy, vz);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int ref_launch_gravity(uint64_t nvox, const int8_t* solids, double* uy, double dt, int remove, cudaStream_t s) {
    if (nvox) ref_gravity_kernel<<<nblk(nvox, 512), 512, 0, s>>>(nvox, solids, uy, dt, remove);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int ref_launch_divergence(uint32_t nodes, const uint32_t* node_voxels, const uint32_t* voxel_ids, const double* ux,
                          const double* uy, const double* uz, const flip_grid& g, const uint32_t* ytable,
                          const uint32_t* starts, const uint32_t* keys, double* divU, cudaStream_t s) {
    if (nodes)
        ref_divergence_kernel<<<nodes, kNodeThreads, 0, s>>>(nodes, node_voxels, voxel_ids, ux, uy, uz, g, ytable, starts,
                                                             keys, divU);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int ref_launch_gs(uint32_t nodes, const uint32_t* node_voxels, const uint32_t* voxel_ids, const int8_t* solids,
                  const double* divU, double* p, double* res, double scale, double w, uint32_t iters, cudaStream_t s) {
    if (nodes && iters)
        ref_gs_kernel<<<nodes, kNodeThreads, 0, s>>>(nodes, node_voxels, voxel_ids, solids, divU, p, res, scale, w, iters);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int ref_launch_velocity_update(uint32_t nodes, const uint32_t* node_voxels, const uint32_t* voxel_ids,
                               const int8_t* solids, const double* p, double* ux, double* uy, double* uz, double scale,
                               cudaStream_t s) {
    if (nodes)
        ref_velocity_update_kernel<<<nodes, kNodeThreads, 0, s>>>(nodes, node_voxels, voxel_ids, solids, p, ux, uy, uz, scale);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}
int ref_launch_getmax_level(uint64_t n, const double* a, double* out, int absolute, cudaStream_t s) {
    uint64_t nb = n / 512 + 1;
    ref_getmax_kernel<<<nblk(nb, 256), 256, 0, s>>>(n, a, out, absolute);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int ref_launch_move_solids(uint32_t nodes, uint64_t n, const uint32_t* starts, const uint32_t* keys, double* px,
                           double* py, double* pz, const uint32_t* node_voxels, const uint32_t* voxel_ids,
                           const int8_t* solids, const flip_grid& g, cudaStream_t s) {
    if (nodes) ref_move_solids_kernel<<<nodes, 32, 0, s>>>(nodes, n, starts, keys, px, py, pz, node_voxels, voxel_ids, solids, g);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int ref_gather_f64(const uint32_t* perm, uint64_t n, const double* in, double* out, cudaStream_t s) {
    if (n) ref_gather_f64_kernel<<<nblk(n, 256), 256, 0, s>>>(perm, n, in, out);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

}  // namespace flip

using namespace flip;

extern "C" int flip_ref_keys(double* px, double* py, double* pz, uint64_t n, const flip_grid* grid, uint32_t* keys,
                             uint32_t* idx, void* stream) {
    if (!grid || (n && (!px || !py || !pz || !keys))) return FLIP_ERR_ARG;
    return ref_launch_keys(px, py, pz, n, *grid, keys, idx, as_stream(stream));
}
extern "C" int flip_ref_ydim_rows(const uint32_t* starts, const uint32_t* sorted_keys, uint32_t nodes,
                                  const flip_grid* grid, uint32_t* table, void* stream) {
    if (!grid || !table) return FLIP_ERR_ARG;
    return ref_launch_ydim(starts, sorted_keys, nodes, *grid, table, as_stream(stream));
}
extern "C" int flip_ref_voxel_counts(const uint32_t* starts, const uint32_t* sorted_keys, uint32_t nodes, uint64_t n,
                                     const double* px, const double* py, const double* pz, const flip_grid* grid,
                                     uint32_t* counts, uint32_t* masks, void* stream) {
    if (!grid || (nodes && (!starts || !sorted_keys || !counts || !masks))) return FLIP_ERR_ARG;
    return ref_launch_voxel_counts(starts, sorted_keys, nodes, n, px, py, pz, *grid, counts, masks, as_stream(stream));
}
extern "C" int flip_ref_voxel_ids(const uint32_t* sorted_keys, uint32_t nodes, const uint32_t* masks,
                                  const uint32_t* node_voxels, const flip_grid* grid, uint32_t* voxel_ids, int8_t* solids,
                                  void* stream) {
    if (!grid) return FLIP_ERR_ARG;
    return ref_launch_voxel_ids(sorted_keys, nodes, masks, node_voxels, *grid, voxel_ids, solids, as_stream(stream));
}
extern "C" int flip_ref_p2g(const uint32_t* starts, const uint32_t* sorted_keys, uint32_t nodes, uint64_t n,
                            const double* px, const double* py, const double* pz, const double* vx, const double* vy,
                            const double* vz, const uint32_t* node_voxels, const uint32_t* voxel_ids,
                            const int8_t* solids, const flip_grid* grid, double* ux, double* uy, double* uz,
                            void* stream) {
    if (!grid) return FLIP_ERR_ARG;
    return ref_launch_p2g(starts, sorted_keys, nodes, n, px, py, pz, vx, vy, vz, node_voxels, voxel_ids, solids, *grid, ux,
                          uy, uz, as_stream(stream));
}
extern "C" int flip_ref_g2p(const uint32_t* starts, const uint32_t* sorted_keys, uint32_t nodes, uint64_t n,
                            const double* px, const double* py, const double* pz, const uint32_t* node_voxels,
                            const uint32_t* voxel_ids, const double* ux, const double* uy, const double* uz,
                            const flip_grid* grid, double* vx, double* vy, double* vz, void* stream) {
    if (!grid) return FLIP_ERR_ARG;
    return ref_launch_g2p(starts, sorted_keys, nodes, n, px, py, pz, node_voxels, voxel_ids, ux, uy, uz, *grid, vx, vy, vz,
                          as_stream(stream));
}

extern "C" size_t flip_ref_getmax_scratch_bytes(uint64_t n) { return 2 * sizeof(double) * (n / 512 + 2); }

extern "C" int flip_ref_getmax_f64(const double* data, uint64_t n, int absolute, void* scratch, size_t scratch_bytes,
                                   double* result, void* stream) {
    if (!data || !result || !scratch || scratch_bytes < flip_ref_getmax_scratch_bytes(n)) return FLIP_ERR_ARG;
    cudaStream_t s = as_stream(stream);
    double* b0 = (double*)scratch;
    double* b1 = b0 + (n / 512 + 2);
    int rc = ref_launch_getmax_level(n, data, b0, absolute, s);
    if (rc) return rc;
    for (uint64_t i = n / 512 + 1; i > 1; i = i / 512 + 1) {
        rc = ref_launch_getmax_level(i, b0, b1, absolute, s);
        if (rc) return rc;
        double* t = b0; b0 = b1; b1 = t;
    }
    FLIP_CUDA_TRY(cudaMemcpyAsync(result, b0, sizeof(double), cudaMemcpyDeviceToHost, s));
    FLIP_CUDA_TRY(cudaStreamSynchronize(s));
    return FLIP_OK;
}
