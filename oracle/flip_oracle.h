/*
 * flip_oracle.h -- CPU restatement of the flip2 fluid step, used ONLY as test
 * infrastructure: the parity checker for the CUDA path and the timed CPU
 * baseline.  Nothing in the product library links or calls this code.
 *
 * Two families of functions:
 *   orc_ref_*   restate the reference engine's kernels stage by stage in FP64
 *               (the reference keeps all particle/grid state in double),
 *               including its documented quirks, so that integer outputs
 *               (keys, permutation, prefix sums, compaction) are bit-exact and
 *               floating-point outputs agree to rounding.
 *   orc_nat_*   the native-mode step (trilinear MAC P2G/G2P, FLIP blend, RK2,
 *               Jacobi-PCG) in FP64: no reference counterpart; the FP64 check
 *               for the FP32 CUDA path.
 *
 * Parity pinning: the reference publishes no golden vectors.  The restatement
 * is pinned against outputs of the reference itself, built from its own
 * sources (oracle/Makefile -> oracle/_ref) and run on a B200 by
 * tests/golden/make_golden.py; the fixtures live in tests/golden/.
 */
#ifndef FLIP_ORACLE_H
#define FLIP_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Mirrors class Grid (engine/grid.hpp:8-38): float corner, uint root-cell
 * counts, float root-cell size. */
typedef struct {
    float negX, negY, negZ;
    uint32_t sizeX, sizeY, sizeZ;
    float cellSize;
} orc_grid;

/* ---------------------------------------------------------------- binning */
/* rootCell (engine/algorithms/particleToGridFunctions.cu:19-45): clamp into
 * the box (in place) and compute the linear root-cell key. */
void orc_ref_keys(int64_t n, double* px, double* py, double* pz, orc_grid g, uint32_t* keys);
/* Stable LSD sort of (key, index) pairs, the semantics of cudaRadixSortUint
 * (engine/algorithms/radixSortKernels.cu:85-123): keys_out sorted, perm with
 * keys_out[j] = keys_in[perm[j]]. */
void orc_sort_pairs(int64_t n, const uint32_t* keys_in, uint32_t* keys_out, uint32_t* perm_out);
/* Same, generic payload: vals_out[j] = vals_in[perm[j]]. */
void orc_sort_pairs_payload(int64_t n, const uint32_t* keys_in, const uint32_t* vals_in,
                            uint32_t* keys_out, uint32_t* vals_out);
/* Inclusive scan, cudaParallelPrefixSum (parallelPrefixSumKernels.cu:54-77). */
void orc_inclusive_scan(int64_t n, uint32_t* a);
/* Exclusive block scan of a 512-voxel tile (parallelPrefixSumKernels.hu:16-48). */
uint32_t orc_exclusive_scan_small(uint32_t n, uint32_t* a);
/* reorderGridIndices<double> (radixSortKernels.cu:59-68). */
void orc_gather_f64(int64_t n, const uint32_t* perm, const double* in, double* out);
/* markUniqueGridCells + inclusive scan (particleToGridFunctions.cu:303-327);
 * returns the number of occupied root cells. */
uint32_t orc_mark_unique_scan(int64_t n, const uint32_t* sorted_keys, uint32_t* flags_scan);
/* mapNodeIndicesToParticles (particleToGridFunctions.cu:329-341). */
void orc_cell_starts(int64_t n, const uint32_t* flags_scan, uint32_t* starts);
/* zeroYDimArray + getYDimPositionFirstInRow (particleToGridFunctions.cu:347-378);
 * the table has sizeY*sizeZ entries, all initialised to nodes. */
void orc_ydim_rows(uint32_t nodes, const uint32_t* starts, const uint32_t* keys, orc_grid g, uint32_t* table);
/* getNumberVoxelsUsedPerNode (engine/particles.cu:88-190): per-node count of
 * used voxels of the 8^3 tile (not yet scanned). */
void orc_ref_voxel_counts(uint32_t nodes, int64_t n, const uint32_t* starts, const uint32_t* keys,
                          const double* px, const double* py, const double* pz, orc_grid g, uint32_t* counts);
/* generateVoxelIDs (engine/particles.cu:192-321); node_voxels is the inclusive
 * scan of the counts. */
void orc_ref_voxel_ids(uint32_t nodes, int64_t n, const uint32_t* starts, const uint32_t* keys,
                       const double* px, const double* py, const double* pz, orc_grid g,
                       const uint32_t* node_voxels, uint32_t* voxel_ids, int8_t* solids);

/* ------------------------------------------------------ reference P2G/G2P */
/* gatherParticleVelsToVoxels (engine/particles.cu:379-488) for one axis
 * (dim 0=X,1=Y,2=Z), weight sums starting from zero. */
void orc_ref_p2g(uint32_t nodes, int64_t n, const uint32_t* starts, const uint32_t* keys,
                 const double* px, const double* py, const double* pz, const double* vdim,
                 const uint32_t* node_voxels, const uint32_t* voxel_ids, const int8_t* solids,
                 orc_grid g, int dim, double* voxel_u);
/* gatherVoxelVelsToParticles (engine/particles.cu:562-662) for one axis. */
void orc_ref_g2p(uint32_t nodes, int64_t n, const uint32_t* starts, const uint32_t* keys,
                 const double* px, const double* py, const double* pz,
                 const uint32_t* node_voxels, const uint32_t* voxel_ids, const double* voxel_u,
                 orc_grid g, int dim, double* vdim);
/* advectParticlePositions (engine/particles.cu:664-669). */
void orc_ref_advect(int64_t n, double dt, double* pos, const double* v);
/* moveSolids (engine/particles.cu:674-740), deterministic part: for each
 * particle that must be re-seeded returns the chosen local voxel id in
 * new_voxel[i] (or UINT32_MAX when it stays).  The random offsets come from
 * the curand device API and are not restated. */
void orc_ref_move_solids_targets(uint32_t nodes, int64_t n, const uint32_t* starts, const uint32_t* keys,
                                 const double* px, const double* py, const double* pz,
                                 const uint32_t* node_voxels, const uint32_t* voxel_ids, const int8_t* solids,
                                 orc_grid g, uint32_t* new_voxel);

/* -------------------------------------------------- reference pressure */
/* CudaVec<double>::getMax (engine/cudaVec.cu:173-233), including its
 * reduction that compares element t with t+256 only. */
double orc_ref_getmax(int64_t n, const double* a, int absolute);
/* applyGravityKernel / removeGravityKernel (voxelSolveFunctions.cu:160-185). */
void orc_ref_gravity(int64_t nvox, const int8_t* solids, double* uy, double dt, int remove);
/* cudaCalcDivU (voxelSolveFunctions.cu:97-271), all three axes. */
void orc_ref_divergence(uint32_t nodes, const uint32_t* node_voxels, const uint32_t* voxel_ids,
                        const double* ux, const double* uy, const double* uz, orc_grid g,
                        const uint32_t* ytable, const uint32_t* starts, const uint32_t* keys, double* divU);
/* One GSiteration launch (voxelSolveFunctions.cu:293-389). */
void orc_ref_gs_pass(uint32_t nodes, const uint32_t* node_voxels, const uint32_t* voxel_ids,
                     const int8_t* solids, const double* divU, double* p, double* res,
                     double density, double dt, orc_grid g, int red, double w);
/* cudaGSiteration (voxelSolveFunctions.cu:391-412); returns the terminating
 * residual and the number of red+black iterations in *iters. */
double orc_ref_gs_solve(uint32_t nodes, const uint32_t* node_voxels, const uint32_t* voxel_ids,
                        const int8_t* solids, const double* divU, double* p, double* res,
                        double density, double dt, orc_grid g, double threshold, uint32_t max_iter,
                        uint32_t* iters);
/* pressureToAcceleration (voxelSolveFunctions.cu:415-479), all three axes. */
void orc_ref_velocity_update(uint32_t nodes, const uint32_t* node_voxels, const uint32_t* voxel_ids,
                             const int8_t* solids, const double* p, double* ux, double* uy, double* uz,
                             double dt, double density, orc_grid g);

/* Whole reference sub-step on host arrays (Particles::solveFrame body,
 * engine/particles.cu:784-803, without moveSolids): rebin, P2G, pressure,
 * velocity update, G2P, advect.  Positions/velocities in/out; returns dt
 * used.  Scratch is allocated internally.  Used as the timed CPU baseline. */
typedef struct {
    uint32_t nodes, voxels, gs_iters_total;
    double dt, residual;
} orc_ref_step_info;
int orc_ref_substep(int64_t n, double* px, double* py, double* pz, double* vx, double* vy, double* vz,
                    orc_grid g, double frameDt, double elapsedThisFrame, int permute_velocities,
                    orc_ref_step_info* info);

/* ----------------------------------------------- native-mode step (FP64) */
typedef struct {
    /* voxel grid: nx*ny*nz cells of size h, origin (ox,oy,oz) */
    double ox, oy, oz, h;
    int32_t nx, ny, nz;
    double gravity_y, flip, dt, tol;
    int32_t max_iter;
    /* velocity of the interior solid cells: faces between a solid and a
     * non-solid cell take it; faces on the box walls stay 0 */
    double solid_u, solid_v, solid_w;
} orc_nat_params;

/* Tile key of each particle (8^3-voxel tiles, x-fastest tile order). */
void orc_nat_keys(int64_t n, const float* pos /*xyz interleaved*/, const orc_nat_params* P, uint32_t* keys);
/* Full native-mode step on interleaved float3 positions/velocities (n*3).
 * solid: optional per-cell solid mask (nx*ny*nz, x fastest) or NULL.
 * Outputs the face grids after P2G (u_p2g, v_p2g, w_p2g; sizes nx*ny*nz,
 * face (i,j,k) = negative face of cell (i,j,k)), the pressure (phi),
 * the PCG iteration count and final relative residual; updates pos/vel. */
typedef struct {
    int32_t iters;
    double rel_residual;
    int64_t fluid_cells;
} orc_nat_info;
int orc_nat_step(int64_t n, float* pos, float* vel, const uint8_t* solid, const orc_nat_params* P,
                 double* u_p2g, double* v_p2g, double* w_p2g, double* phi, orc_nat_info* info);
/* The same step, also writing the face grids after the projection (u_proj,
 * v_proj, w_proj; any may be NULL): the grid velocity G2P samples. */
int orc_nat_step_ex(int64_t n, float* pos, float* vel, const uint8_t* solid, const orc_nat_params* P,
                    double* u_p2g, double* v_p2g, double* w_p2g, double* phi, double* u_proj, double* v_proj,
                    double* w_proj, orc_nat_info* info);
/* Individual pieces, for stage-level checks. */
void orc_nat_p2g(int64_t n, const float* pos, const float* vel, const orc_nat_params* P,
                 double* u, double* v, double* w, uint8_t* fluid);
/* Jacobi-PCG on the 7-point system of the cell types (0 air,1 fluid,2 solid):
 * A x = b over fluid cells; returns iterations. */
int orc_nat_pcg(const uint8_t* type, const double* b, double* x, const orc_nat_params* P, double* rel_res);
/* Apply the 7-point operator (for residual checks). */
void orc_nat_apply_A(const uint8_t* type, const double* x, double* y, const orc_nat_params* P);

/* Learned pressure preconditioner (no reference counterpart): grids x
 * fastest, weights [27 taps][Cin][Cout] per layer (3->16->16->16->1). */
int orc_lp_num_weights(void);
void orc_lp_forward(int nx, int ny, int nz, const uint8_t* type, const float* r, const float* w, const int* dil,
                    int round_bf16, float* z, double* inv_s);
double orc_lp_loss_grad(int nx, int ny, int nz, const uint8_t* type, const float* r, const float* e, const float* w,
                        const int* dil, int round_bf16, float* z, double* grad);
int orc_lp_fpcg(int nx, int ny, int nz, const uint8_t* type, const double* b, const float* w, const int* dil,
                int round_bf16, double tol, int max_iter, double* x, double* rel_res);

/* Multilevel preconditioner (pressure_method 2, no reference counterpart):
 * levels of the hierarchy below an nx x ny x nz grid (padded dims of each
 * level into dims[3 l ..]), one V-cycle z = M(r) (mode 0: the network solves
 * the coarsest level, 1: Jacobi sweeps only), and FCG with it. */
int orc_mg_levels(int nx, int ny, int nz, int* dims);
void orc_mg_apply(int nx, int ny, int nz, const uint8_t* type, const float* r, const float* w, const int* dil,
                  int round_bf16, int mode, double* z);
int orc_mg_fcg(int nx, int ny, int nz, const uint8_t* type, const double* b, const float* w, const int* dil,
               int round_bf16, int mode, double tol, int max_iter, double* x, double* rel_res);

#ifdef __cplusplus
}
#endif
#endif
