// native.cuh -- declarations shared by native.cu and the engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace flip {

// cell types
constexpr uint8_t kAir = 0, kFluid = 1, kSolid = 2;

// voxel grid of the native-mode step: nx*ny*nz voxels (multiples of 8) of size
// h, tiles of 8^3 voxels
struct NatDims {
    int nx, ny, nz;
    int tx, ty, tz;
    float ox, oy, oz, h;
};

// device-resident Jacobi-PCG state (FP64 scalars)
struct PcgState {
    double bb, rz, rz_prev, pq, rr, rr_true, alpha, beta, tol2;
    int iter, done, pending, max_iter, true_every, true_checks, next_check;
    int pcur;   // which p buffer holds the current direction
    int flush;  // fold xg into x at the next direction update
    unsigned int ticket;
    int halt;   // done || pending: the network and dot kernels of FPCG stop too
    float inv_s;  // 1 / rms(r) over fluid cells: input scale of the learned preconditioner
    int flexible; // 1: FPCG (z = N(r) given), 0: Jacobi PCG
    double zq, nfluid;
    int chunks;   // chunks the device-side loop has run
    double rr_check;  // r.r at the previous true-residual check (bb before the first)
};
// flexible CG gives up (done = 4) when the true r.r at a check exceeds this
// fraction of the previous check's: the residual norm fell by less than 10%
constexpr double kFlexStall = 0.81;

constexpr int kPcgBlocks = 592;        // 148 SMs x 4 CTAs of 512 threads
constexpr int kPcgUpdateBlocks = 592;  // 148 SMs x 4 CTAs of 256 threads (a warp per half tile, 10 loads in flight a lane)

// PCG vectors on the tile-blocked slots.  The solution is x + xg: x in FP64
// holds everything up to the last true-residual check, xg (FP32) the
// increments since then.  An FP32 solution alone bounds the attainable true
// residual near eps_32 * cond(A) (2.5e-5 on the 32^3 dam-break), above the
// 1e-6 target; the FP64 part removes that floor while each iteration moves
// only FP32 data.  At every check r is replaced by b - A(x + xg) computed in
// FP64, and the next direction update folds xg into x.  r, p, q and the stencil
// arithmetic are FP32; every dot product is FP64.
// cell: bit 7 = fluid, bits 0-2 = number of non-solid neighbours (the
// Jacobi diagonal), 0 for every other cell.
struct PcgBuffers {
    double* x;
    float *xg, *b, *r, *p0, *p1, *q, *z;
    uint8_t* cell;
    uint32_t* tcoord;  // packed tile coordinates of the occupied tiles
    PcgState* st;
    double* partials;  // [4][kPcgBlocks]
};
constexpr uint8_t kCellFluid = 0x80;

int nat_launch_keys(const float* px, const float* py, const float* pz, uint64_t n, const NatDims& D, uint32_t* keys,
                    cudaStream_t s);
int nat_launch_gather(const uint32_t* perm, uint64_t n, const float* const* src, float* const* dst, cudaStream_t s);
int nat_launch_p2g(const uint32_t* tile_keys, const uint32_t* starts, const uint32_t* d_ntiles, uint64_t n,
                   const float* const* ps, const float* const* vs, const NatDims& D, float* const* m, float* const* w,
                   uint8_t* type, int grid, cudaStream_t s);
int nat_launch_tile_coords(const uint32_t* tile_keys, const uint32_t* d_ntiles, const NatDims& D, uint32_t* coords,
                           int grid, cudaStream_t s);
int nat_launch_dilate_compact(const uint32_t* tile_keys, const uint32_t* d_ntiles, const NatDims& D, uint8_t* flags,
                              uint32_t* list, uint32_t* d_count, int grid, cudaStream_t s);
int nat_launch_poisson_gen(const NatDims& D, float surface, const float4* sph, int nsph, const float* imp, int nimp,
                           float gdt, uint8_t* type, float* b, uint64_t nslots, cudaStream_t s);
int nat_launch_fluid_tiles(const uint8_t* type, uint8_t* flags, uint32_t ntiles_total, uint32_t* list, uint32_t* d_count,
                           uint64_t nslots, cudaStream_t s);
int nat_launch_lin_tiles_f32(const float* src, float* dst, const NatDims& D, int to_tiles, cudaStream_t s);
// x = x + xg on the fluid cells of the last solve (0 elsewhere), xg = 0
int nat_launch_fold_pressure(double* x, float* xg, const uint8_t* cell, uint64_t nslots, cudaStream_t s);
int nat_launch_solution_lin(const double* x, const float* xg, const uint8_t* cell, const NatDims& D, double* out,
                            cudaStream_t s);
int nat_launch_apply_solids(const uint8_t* solid, uint8_t* type, uint64_t nslots, cudaStream_t s);
int nat_launch_mask_to_tiles(const uint8_t* lin, const NatDims& D, uint8_t* tiled, cudaStream_t s);
// P2G sums -> face velocities; gravity on faces touching fluid; wall faces
// 0; faces between a solid and a non-solid cell take usolid
int nat_launch_normalize(const uint32_t* tiles, const uint32_t* d_count, const NatDims& D, float gdt, float* const* m,
                         const float* const* w, float* const* o, const uint8_t* type, float3 usolid, int grid,
                         cudaStream_t s);
// U == nullptr: the right-hand side is already in B.b (standalone Poisson problems).
// cell_prev != nullptr: warm start from the previous solution (x + xg) on the
// cells that were fluid in the previous solve (cell_prev: its cell codes)
int nat_launch_pcg_init(const uint32_t* tiles, const uint32_t* d_ntiles, const NatDims& D, const float* const* U,
                        const uint8_t* type, PcgBuffers& B, cudaStream_t s, const uint8_t* cell_prev = nullptr);
// flexible PCG: direction from z (B.z), and the r.z / z.q reduction giving beta
int nat_launch_fpcg_direction_update(const uint32_t* tiles, const uint32_t* d_ntiles, const NatDims& D, PcgBuffers& B,
                                     cudaStream_t s);
// jacobi = 1 adds D^-1 r to z first (the network preconditioner's Jacobi
// term); the multilevel preconditioner's z is complete (jacobi = 0)
int nat_launch_fpcg_dot(const uint32_t* tiles, const uint32_t* d_ntiles, PcgBuffers& B, int init, cudaStream_t s,
                        int jacobi = 1);
// one PCG iteration: fused direction update + matvec (+ p.Ap), then the
// x/r update (+ r.r, r.z); the two p buffers alternate under device control
int nat_launch_pcg_iteration(const uint32_t* tiles, const uint32_t* d_ntiles, const NatDims& D, PcgBuffers& B,
                             cudaStream_t s);
// true residual r = b - A x in FP64 when convergence is claimed or every
// true_every iterations; decides convergence
int nat_launch_pcg_check(const uint32_t* tiles, const uint32_t* d_ntiles, const NatDims& D, PcgBuffers& B,
                         cudaStream_t s);
// end of a loop chunk inside a conditional WHILE graph node: continue while
// the solve is not done and fewer than limit chunks have run
int nat_launch_loop_ctl(cudaGraphConditionalHandle h, PcgState* st, int limit, cudaStream_t s);
// *d_out = bits of max over particles of max(|vx|, |vy|, |vz|) (the Courant limit's speed)
int nat_launch_vmax(uint64_t n, const float* const* V, uint32_t* d_out, int grid, cudaStream_t s);
int nat_launch_project(const uint32_t* tiles, const uint32_t* d_count, const NatDims& D, const double* phi,
                       const float* phig, const uint8_t* type, float* const* U, int grid, cudaStream_t s);
int nat_launch_g2p(uint64_t n, const NatDims& D, float dt, float flip, const float* const* U, const float* const* O,
                   float* const* P, float* const* V, cudaStream_t s);

}  // namespace flip
