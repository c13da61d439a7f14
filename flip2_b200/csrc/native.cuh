// native.cuh -- declarations shared by native.cu and the engine.
#pragma once
#include <cuda.h>
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
    float inv_h;  // 1 / h: a position maps to grid coordinates as (p - o) * inv_h wherever cells, keys and stencils are taken
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
    // device flag of the warm start (optional): the previous solve converged,
    // so its solution may start this one; 0 makes a warm-start launch cold
    const int* warm_ok;
};

// Outcome of the last pressure solve, kept on the device so that steps and
// frames captured in a CUDA graph need no host round trip; the host reads
// it when asked (flip_get_info, flip_get_solve_info).
struct SolveRecord {
    int iters;          // iterations of the method asked for
    int plain_iters;    // iterations of a Jacobi-PCG restart (0 if none)
    int converged;      // the true relative residual met tol
    int fell_back;      // the flexible solve missed tol and Jacobi-PCG restarted
    double rel_residual;
    int warm_ok;        // converged: the next step may start from this pressure
    int pad;
    unsigned long long solves, fallbacks;        // since the counters were last cleared
    unsigned long long iters_total;              // iterations of every solve, restarts included
    unsigned long long chunks_primary, chunks_plain;  // loop chunks run in captured solves (the launch count)
    unsigned long long fallbacks_captured;           // restarts inside captured solves (the launch count)
};

// Sub-step control of a captured frame: the device picks each sub-step's dt.
struct FrameState {
    double t;           // time already taken in this frame
    double frame_dt;    // length of the frame
    double max_dt;      // largest sub-step
    double h;           // voxel size (the Courant limit is 0.7 h / max |v|)
    float dt, gdt;      // this sub-step's dt and gravity * dt, read by the step's kernels
    int substeps;
    int error;          // 1: dt collapsed (the frame stopped)
};
constexpr uint8_t kCellFluid = 0x80;

// The last CTA to finish sums the per-CTA partials, in CTA order (deterministic
// for a given grid of at most kPcgBlocks CTAs of NT threads); out[] valid in
// thread 0 of that CTA.
template <int NV, int NT>
__device__ __forceinline__ bool last_block_reduce_n(double (&v)[NV], double* partials, unsigned int* ticket, double* sh,
                                                    double (&out)[NV]) {
    __shared__ bool s_last;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double r = block_sum_f64<NT>(v[q], sh);
        if (threadIdx.x == 0) partials[q * kPcgBlocks + blockIdx.x] = r;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double a = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += NT) a += ((volatile double*)partials)[q * kPcgBlocks + b];
        out[q] = block_sum_f64<NT>(a, sh);
    }
    if (threadIdx.x == 0) *ticket = 0u;
    return true;  // out[] valid in thread 0
}

// TMA descriptor of an arbitrary dense tensor (rank <= 5, strides in bytes of
// dims 1 .. rank-1), zero fill outside it
int encode_tensor_map(CUtensorMap* map, CUtensorMapDataType dtype, int rank, const void* base, const uint64_t* dims,
                      const uint64_t* strides_bytes, const uint32_t* box);

int nat_launch_keys(const float* px, const float* py, const float* pz, uint64_t n, const NatDims& D, uint32_t* keys,
                    cudaStream_t s);
int nat_launch_gather(const uint32_t* perm, uint64_t n, const float* const* src, float* const* dst, cudaStream_t s);
// occupied tiles of sorted tile keys, in key order: list[c] the tile key,
// starts[c] its first particle, *d_count their number, from the sort's head
// table (dense[key] = the first particle of the tile, 0xFFFFFFFF for an
// empty tile; ntiles_total words)
int nat_launch_segment_heads(const uint32_t* dense, uint32_t ntiles_total, uint32_t* list, uint32_t* starts,
                             uint32_t* d_count, cudaStream_t s);
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
// lin / lin_old (optional): x-fastest copies of the face velocities and of
// the P2G ("old") velocities, for the TMA boxes of G2P; gdt_p (optional)
// replaces gdt by a device value
int nat_launch_normalize(const uint32_t* tiles, const uint32_t* d_count, const NatDims& D, float gdt, float* const* m,
                         const float* const* w, float* const* o, const uint8_t* type, float3 usolid, int grid,
                         cudaStream_t s, float* const* lin = nullptr, float* const* lin_old = nullptr,
                         const float* gdt_p = nullptr);
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
// the plain solve's form of the above: the residual kept as w = D^-1 r, zero
// (like both direction buffers) on the non-fluid cells of the dilated tile
// list dil_tiles (which nat_launch_pcgw_init walks), so that the matvec
// reads its halo without cell codes; init, iteration and true-residual check
// as nat_launch_pcg_init / _iteration / _check otherwise
int nat_launch_pcgw_init(const uint32_t* tiles, const uint32_t* d_ntiles, const uint32_t* dil_tiles,
                         const uint32_t* d_ndil, const NatDims& D, const float* const* U, const uint8_t* type,
                         PcgBuffers& B, cudaStream_t s, const uint8_t* cell_prev = nullptr);
int nat_launch_pcgw_iteration(const uint32_t* tiles, const uint32_t* d_ntiles, const NatDims& D, PcgBuffers& B,
                              cudaStream_t s);
int nat_launch_pcgw_check(const uint32_t* tiles, const uint32_t* d_ntiles, const NatDims& D, PcgBuffers& B,
                          cudaStream_t s);
// end of a loop chunk inside a conditional WHILE graph node: continue while
// the solve is not done and fewer than limit chunks have run
int nat_launch_loop_ctl(cudaGraphConditionalHandle h, PcgState* st, int limit, cudaStream_t s);
// PcgState for a new solve: tolerance tol^2 of the relative residual,
// iteration cap, FP64 true-residual period, flexible (FCG) or Jacobi-PCG
int nat_launch_state_init(PcgState* st, double tol, int max_iter, int true_every, int flexible, cudaStream_t s);
// the solve's outcome into rec: stage 0 after the method asked for (method 0:
// Jacobi-PCG; else the flexible solve, whose miss of tol is a fallback),
// stage 1 after the Jacobi-PCG restart; captured: the solve ran inside a
// captured step (its loop chunks count towards the step's launches)
int nat_launch_solve_record(SolveRecord* rec, PcgState* st, int flexible, int stage, int captured, cudaStream_t s);
// sets a conditional node's condition value
int nat_launch_cond_set(cudaGraphConditionalHandle h, unsigned int v, cudaStream_t s);
// condition of a conditional IF node: the flexible solve did not converge
int nat_launch_fallback_cond(cudaGraphConditionalHandle h, const PcgState* st, cudaStream_t s);
// one sub-step of a captured frame: dt = min(max_dt, Courant limit from
// *vmax_bits, the rest of the frame) into fs, and the WHILE condition of the
// sub-step loop (more of the frame left after this sub-step)
int nat_launch_frame_ctl(cudaGraphConditionalHandle h, FrameState* fs, const uint32_t* vmax_bits, float gravity_y,
                         cudaStream_t s);
// a new frame of length frame_dt in fs (t = 0, no sub-steps yet)
int nat_launch_frame_init(FrameState* fs, double frame_dt, double max_dt, double h, cudaStream_t s);
// fs->dt and fs->gdt of a fixed-dt step
int nat_launch_step_dt(FrameState* fs, double dt, float gravity_y, cudaStream_t s);
// *d_out = bits of max over particles of max(|vx|, |vy|, |vz|) (the Courant limit's speed)
int nat_launch_vmax(uint64_t n, const float* const* V, uint32_t* d_out, int grid, cudaStream_t s);
// lin (optional): the x-fastest copy of U, updated alike
int nat_launch_project(const uint32_t* tiles, const uint32_t* d_count, const NatDims& D, const double* phi,
                       const float* phig, const uint8_t* type, float* const* U, int grid, cudaStream_t s,
                       float* const* lin = nullptr);
// TMA descriptors of the x-fastest copies of the new (u) and old (o) face
// velocities, encoded once per domain
struct NatG2PMaps {
    CUtensorMap u[3], o[3];
};
int nat_make_g2p_maps(NatG2PMaps& M, float* const* ulin, float* const* olin, const NatDims& D);
// G2P + FLIP blend + RK2 advection per occupied tile (tile_keys/starts of this
// step's binning), grids staged by TMA; particle state read from P, V and
// written to Pout, Vout (the same arrays, or the pre-gather ones); dt_p
// (optional) replaces dt by a device value; keys_out (optional) receives each
// particle's tile key at its new position; solid_type (optional, the cell
// types of this step, tile-blocked): a particle whose new position lies in a
// solid cell keeps its old position and takes the velocity usolid; a TMA
// wait that gives up sets DEVERR_TMA_TIMEOUT in *err
int nat_launch_g2p(const NatG2PMaps& M, const uint32_t* tile_keys, const uint32_t* starts, const uint32_t* d_ntiles,
                   uint64_t n, const NatDims& D, float dt, float flip, const float* const* U, const float* const* O,
                   const float* const* P, const float* const* V, float* const* Pout, float* const* Vout,
                   uint32_t* keys_out, const uint8_t* solid_type, float3 usolid, const float* dt_p, uint32_t* err,
                   int grid, cudaStream_t s);

}  // namespace flip
