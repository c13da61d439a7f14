// mg.cuh -- the multilevel form of the learned pressure preconditioner: one
// V-cycle of damped Jacobi smoothing over a hierarchy of 2x coarsened grids,
// whose coarsest level (16^3 or less) is solved by the 3^3 convolution
// network of lprec.cuh.  No reference counterpart.
//
// Levels.  Level 0 is the solver's grid (its occupied tiles, PCG cell codes).
// Level l+1 has ceil(n_l / 2) cells per axis, padded to whole 8^3 tiles;
// cells past that extent are solid.  The smoothing walks the tiles with
// fluid cells of each level, and every tile of the coarsest (at most 8).
// A coarse cell is air if any of its 8 children is air (the
// Dirichlet condition of the free surface reaches the coarse problem), else
// fluid if any child is fluid, else solid; its operator is the 7-point
// Laplacian of those types on the coarse grid.
//
// V-cycle on level l with right-hand side r (z = output, omega = 2/3):
//   t  = omega D^-1 r, then t += omega D^-1 (r - A t)       (pre-smoothing)
//   r' = R (r - A t),  R = 1/2 x the sum over the 8 children (4 x the average:
//        the coarse operator is the fine one with h doubled)
//   e  = V-cycle(l + 1, r')
//   t += P e  (P: the parent's value, fluid cells only), then two sweeps
//        t += omega D^-1 (r - A t)                          (post-smoothing)
// On the coarsest level z = N(r) + D^-1 r (N: the network) followed by two
// sweeps, or without the network z = omega D^-1 r and the same sweeps (or,
// for comparison, z = a Jacobi-PCG solution in one CTA and the sweeps).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "native.cuh"

namespace flip {

constexpr int kMgMaxLevels = 8;
constexpr int kMgCoarsest = 16;  // coarsen until every axis has at most this many cells
constexpr float kMgOmega = 2.0f / 3.0f;

struct MgLevel {
    NatDims D;              // padded to whole tiles
    int ex, ey, ez;         // cells of the level; past them the grid is solid
    uint32_t ntiles;        // tiles of the level's box
    const uint32_t* tiles;  // tile list: the tiles with fluid cells (the
                            // coarsest level: every tile)
    const uint32_t* d_ntiles;
    uint8_t* type;          // 0 air, 1 fluid, 2 solid
    uint8_t* cell;          // PCG cell code: bit 7 fluid, bits 0-2 non-solid neighbours
    uint8_t* active;        // [tiles] the coarsest level: all 1 (the network's active
                            // flags); intermediate levels: fluid-tile flags
    float* r;               // right-hand side of the level's correction problem
    float* z;               // the level's V-cycle output
    float* t;               // pre-smoothing iterate (read back by the post-smoothing)
};

constexpr int kMgScalePartials = 2048;  // doubles: 2 x the grid of a fused input scale

struct MgHierarchy {
    int levels;
    MgLevel L[kMgMaxLevels];
    float* inv_s;   // 1 / rms of the coarsest right-hand side (the network's input scale)
    float* f0;      // f(0) on the coarsest level
    double* scale_partials;      // kMgScalePartials doubles for the fused input scale
    unsigned int* scale_ticket;  // its last-CTA ticket (0 between launches)
};
// the network's input scale taken by the last down kernel as it writes the
// coarsest right-hand side: 1 / rms over the coarsest fluid cells into inv_s
struct MgScale {
    double* partials;
    unsigned int* ticket;
    float* inv_s;
};

// level dimensions below a fine grid of nx x ny x nz (multiples of 8) cells
int mg_plan(int nx, int ny, int nz, float h, MgLevel* L, int max_levels);
// coarse types and cell codes of every level from level 0's types and
// codes, and the fluid-tile lists of the intermediate levels
int mg_build(const MgHierarchy& H, const int* halt, cudaStream_t s);
// one V-cycle up to the coarsest level's input: smoothing and restriction
// on levels 0 .. levels-2, one kernel per level (the coarsest right-hand
// side ends in L[levels-1].r); scale: the last kernel also sets *H.inv_s as
// mg_input_scale does (at least two levels)
int mg_down(const MgHierarchy& H, const int* halt, int grid0, cudaStream_t s, bool scale = false);
// the coarsest level's solve around a network output zn (nullptr: no
// network): z = zn + D^-1 r (or omega D^-1 r), then two sweeps (one kernel);
// solved: zn is already a coarse solution (z = zn, then the sweeps)
int mg_coarsest(const MgHierarchy& H, const float* zn, const int* halt, cudaStream_t s, bool solved = false);
// FCG's dot products taken by level 0's post-smoothing as it writes z:
// r.z and z.q over the fluid cells, then beta = -z.q / p.q (0 when init) and
// the state's rz, rz_prev, zq -- what fpcg_dot_kernel does without the
// Jacobi term.  partials: 2 x the level-0 grid doubles.
struct MgDot {
    const float* q;
    PcgState* st;
    double* partials;
    int init;
};
// prolongation and post-smoothing back up to level 0, one kernel per level
// (the output in L[0].z); dot: fuse FCG's dot products into the last kernel
int mg_up(const MgHierarchy& H, const int* halt, int grid0, cudaStream_t s, const MgDot* dot = nullptr);
// x = A^-1 b on level L by Jacobi-PCG in one CTA (|r| <= tol |b| or
// max_iter iterations; *iters = iterations run); r, p, q: scratch of the
// level's size
int mg_cg(const MgLevel& L, const float* b, float* x, float* r, float* p, float* q, double tol, int max_iter, int* iters,
          cudaStream_t s, const int* halt = nullptr);
// *inv_s = 1 / rms(r) over the fluid cells of the coarsest level (one CTA)
int mg_input_scale(const MgHierarchy& H, const int* halt, cudaStream_t s);

}  // namespace flip
