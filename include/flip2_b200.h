/*
 * flip2_b200.h -- C ABI of libflip2_b200.so, a B200 (sm_100a) PIC/FLIP fluid
 * step that can stand in for the flip2 engine library (libparticles.so).
 *
 * Two layers:
 *   1. Primitive entry points on caller-owned device memory (plain pointers,
 *      sizes and a cudaStream_t passed as void*).  Each replaces one host
 *      wrapper of the reference's kernel library; the citation names it.
 *      Those that need scratch take it from the caller: query the size with
 *      the matching *_scratch_bytes() function.
 *   2. An engine handle (flip_*) that owns all particle and grid state and
 *      mirrors the reference's Particles class (engine/particles.hu:11-95):
 *      setDomain, initialize, solveFrame and the per-stage methods.
 *
 * All functions return a flip_status; none of them exits the process (the
 * reference's gpuErrchk calls exit(), engine/typedefs.h:12-20).  Device
 * pointers are never freed by the library unless it allocated them.
 */
#ifndef FLIP2_B200_H
#define FLIP2_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    FLIP_OK = 0,
    FLIP_ERR_ARG = 1,           /* bad argument or size                       */
    FLIP_ERR_CUDA = 2,          /* a CUDA runtime call failed                 */
    FLIP_ERR_OOM = 3,           /* device allocation failed                   */
    FLIP_ERR_TIMEOUT = 4,       /* a bounded device wait gave up              */
    FLIP_ERR_STATE = 5,         /* call out of order (e.g. step before init)  */
    FLIP_ERR_NOT_CONVERGED = 6, /* pressure solve hit its iteration cap       */
    FLIP_ERR_DEVICE = 7         /* no usable sm_100 device                    */
} flip_status;

/* Domain descriptor, field for field the reference's Grid
 * (engine/grid.hpp:8-38): float corner, uint root-cell counts, float
 * root-cell size.  A root cell holds 4x4x4 voxels. */
typedef struct {
    float negX, negY, negZ;
    uint32_t sizeX, sizeY, sizeZ;
    float cellSize;
} flip_grid;

/* Library version and the status string of the last failure on this thread. */
const char* flip_version(void);
const char* flip_status_string(int status);
/* Architecture of the device code the runtime loaded for this library
 * (cudaFuncAttributes::binaryVersion of its scan kernel): 100 for sm_100a.
 * Needs a visible device.  No reference counterpart. */
int flip_binary_version(int* version);

/* ------------------------------------------------------------------ */
/* 1. Primitives                                                       */
/* ------------------------------------------------------------------ */

/* rootCell + cudaFindGridCell (engine/algorithms/particleToGridFunctions.cu:19-45,216-219):
 * clamp FP64 positions into the box in place and write the linear root-cell
 * key x + y*sizeX + z*sizeX*sizeY of each particle.  If idx != NULL also
 * writes idx[i] = i (the sort payload). */
int flip_ref_keys(double* px, double* py, double* pz, uint64_t n, const flip_grid* grid,
                  uint32_t* keys, uint32_t* idx, void* stream);

/* Stable LSD radix sort of (u32 key, u32 value) pairs, 8-bit digits,
 * onesweep passes with decoupled look-back.  Replaces cudaRadixSortUint /
 * cudaSortParticlesByGridNode (engine/algorithms/radixSortKernels.cu:85-123,
 * particleToGridFunctions.cu:270-301): with vals_in == NULL the payload is
 * the index, so vals_out is the reference's reorderedGridIndices
 * (keys_out[j] == keys_in[vals_out[j]]).  key_bits (1..32) bounds the keys:
 * every key must be < 2^key_bits.  keys_in may equal keys_out. */
size_t flip_sort_pairs_scratch_bytes(uint64_t n);
int flip_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out, uint32_t* vals_out,
                    uint64_t n, int key_bits, void* scratch, size_t scratch_bytes, void* stream);

/* Inclusive prefix sum of u32 (wrapping), single pass with decoupled
 * look-back.  Replaces cudaParallelPrefixSum
 * (engine/algorithms/parallelPrefixSumKernels.cu:54-77).  In place allowed. */
size_t flip_inclusive_scan_scratch_bytes(uint64_t n);
int flip_inclusive_scan_u32(const uint32_t* in, uint32_t* out, uint64_t n, void* scratch, size_t scratch_bytes,
                            void* stream);

/* flip_inclusive_scan_u32 for callers that cannot allocate device memory
 * (no counterpart in the reference): the look-back scratch is a static
 * device array of the library (512 KiB per GPU, held until exit), so only
 * in and out are passed.  n <= 2^28, else FLIP_ERR_ARG.  Calls share that
 * array: calls that overlap on the GPU race and must be serialised.  The
 * first call on each device resolves the array's address; make it before any
 * stream capture (a failed lookup is retried by the next call).  The call
 * returns before its kernel runs, so a look-back wait that gives up is
 * reported by flip_inclusive_scan_u32_noalloc_status, not by this call. */
int flip_inclusive_scan_u32_noalloc(const uint32_t* in, uint32_t* out, uint64_t n, void* stream);
/* Companion of flip_inclusive_scan_u32_noalloc (no counterpart in the
 * reference; allocates nothing): waits for `stream`, then copies the static
 * array's error word of the last call on the current device into *flags.
 * Returns FLIP_ERR_TIMEOUT when bit 0 (a look-back wait gave up) is set: that
 * call's output is invalid. */
int flip_inclusive_scan_u32_noalloc_status(void* stream, uint32_t* flags);

/* Device status of the last flip_sort_pairs, flip_inclusive_scan_u32 or
 * flip_segment_heads call that used `scratch` (no reference counterpart: the
 * reference's kernels have no failure word).  Waits for `stream`, then copies
 * the scratch's first word into *flags.  Bit 0 means a decoupled look-back
 * wait gave up after its poll limit (the kernel returned, but its output is
 * invalid): FLIP_ERR_TIMEOUT is returned. */
int flip_scratch_status(const void* scratch, void* stream, uint32_t* flags);
/* Test hook for those bounded waits (no reference counterpart): the scan
 * (which = 0, out_keys receives the scan) or the sort with the index payload
 * (which = 1, 32-bit keys) of more keys than one tile holds (4096 for the
 * scan, 6144 for the sort) from `in`, run with tile 0 never
 * claimed, so that tile 1's look-back polls a word nothing publishes and
 * gives up after spin_limit polls.  Returns flip_scratch_status's result:
 * FLIP_ERR_TIMEOUT with bit 0 in *flags.  The outputs are invalid; the
 * context stays usable. */
int flip_test_lookback_timeout(int which, const uint32_t* in, uint32_t* out_keys, uint32_t* out_vals, uint64_t n,
                               uint32_t spin_limit, void* scratch, size_t scratch_bytes, void* stream,
                               uint32_t* flags);

/* Segment heads of sorted keys, fused: replaces cudaMarkUniqueGridCellsAndCount
 * + cudaMapNodeIndicesToParticles (particleToGridFunctions.cu:303-345).
 * flags_scan (optional) receives the inclusive scan of the head flags
 * (the reference's uniqueGridNodeIndices), starts[k] the first index of the
 * k-th distinct key, node_keys[k] (optional) that key, *d_count (device) the
 * number of distinct keys.  starts must hold up to n entries. */
size_t flip_segment_heads_scratch_bytes(uint64_t n);
int flip_segment_heads(const uint32_t* sorted_keys, uint64_t n, uint32_t* flags_scan, uint32_t* starts,
                       uint32_t* node_keys, uint32_t* d_count, void* scratch, size_t scratch_bytes, void* stream);

/* zeroYDimArray + getYDimPositionFirstInRow (particleToGridFunctions.cu:347-378):
 * table[sizeY*sizeZ] of the first root-cell id of each (y,z) row, every
 * entry initialised to `nodes`. */
int flip_ref_ydim_rows(const uint32_t* starts, const uint32_t* sorted_keys, uint32_t nodes, const flip_grid* grid,
                       uint32_t* table, void* stream);

/* getNumberVoxelsUsedPerNode (engine/particles.cu:88-190): per occupied
 * root cell, the number of used voxels of its 8^3 tile, plus the tile's
 * 512-bit used mask (64 bytes per node) reused by flip_ref_voxel_ids. */
int flip_ref_voxel_counts(const uint32_t* starts, const uint32_t* sorted_keys, uint32_t nodes, uint64_t n,
                          const double* px, const double* py, const double* pz, const flip_grid* grid,
                          uint32_t* counts, uint32_t* masks, void* stream);
/* generateVoxelIDs (engine/particles.cu:192-321) from the masks and the
 * inclusive scan of the counts (nodeIndexUsedVoxels). */
int flip_ref_voxel_ids(const uint32_t* sorted_keys, uint32_t nodes, const uint32_t* masks,
                       const uint32_t* node_voxels, const flip_grid* grid, uint32_t* voxel_ids, int8_t* solids,
                       void* stream);

/* gatherParticleVelsToVoxels for the three axes in one launch
 * (engine/particles.cu:379-505), FP64, weight sums zero-initialised. */
int flip_ref_p2g(const uint32_t* starts, const uint32_t* sorted_keys, uint32_t nodes, uint64_t n,
                 const double* px, const double* py, const double* pz,
                 const double* vx, const double* vy, const double* vz,
                 const uint32_t* node_voxels, const uint32_t* voxel_ids, const int8_t* solids,
                 const flip_grid* grid, double* ux, double* uy, double* uz, void* stream);

/* gatherVoxelVelsToParticles for the three axes (engine/particles.cu:562-662,742-749). */
int flip_ref_g2p(const uint32_t* starts, const uint32_t* sorted_keys, uint32_t nodes, uint64_t n,
                 const double* px, const double* py, const double* pz,
                 const uint32_t* node_voxels, const uint32_t* voxel_ids,
                 const double* ux, const double* uy, const double* uz, const flip_grid* grid,
                 double* vx, double* vy, double* vz, void* stream);

/* CudaVec<double>::getMax(stream, abs) (engine/cudaVec.cu:173-233) with the
 * reference's reduction, which compares element t with t+256 of each
 * 512-element block only; synchronous, result written to *result (host). */
size_t flip_ref_getmax_scratch_bytes(uint64_t n);
int flip_ref_getmax_f64(const double* data, uint64_t n, int absolute, void* scratch, size_t scratch_bytes,
                        double* result, void* stream);

/* ------------------------------------------------------------------ */
/* 2. Engine handle (mirrors class Particles)                          */
/* ------------------------------------------------------------------ */

typedef struct flip_engine flip_engine;

typedef enum {
    FLIP_MODE_REFERENCE = 0, /* the reference's math: FP64 state, tent P2G/G2P, PIC,
                                forward Euler, tile-local red-black SOR            */
    FLIP_MODE_NATIVE = 1     /* FP32 state, trilinear MAC P2G/G2P, FLIP blend, RK2,
                                matrix-free Jacobi-PCG with FP64 reductions        */
} flip_mode;

typedef struct {
    int32_t mode;                /* flip_mode                                       */
    float flip_ratio;            /* NATIVE: FLIP/PIC blend (0.95)                   */
    float gravity_y;             /* NATIVE: -9.8                                    */
    double pcg_tol;              /* NATIVE: relative residual target (1e-6)         */
    int32_t pcg_max_iter;        /* NATIVE: iteration cap                           */
    int32_t pcg_check_every;     /* NATIVE: iterations between convergence reads    */
    int32_t true_residual_every; /* NATIVE: FP64 r = b - A x recomputation period   */
    int32_t permute_velocities;  /* REFERENCE: 0 = keep the reference's order (Q5)  */
    int32_t device;              /* CUDA device ordinal                             */
    int32_t pressure_method;     /* NATIVE: 0 Jacobi-PCG; 1 FPCG preconditioned by the
                                    network on the solver's grid; 2 FPCG preconditioned
                                    by a multigrid V-cycle whose coarsest level (16^3 or
                                    less) the network solves                          */
    double max_substep_dt;       /* NATIVE: largest sub-step of solveFrame (1/240)  */
    int32_t learned_max_iter;    /* NATIVE: FPCG cap before the Jacobi-PCG restart   */
    int32_t lp_cuda_cores;       /* NATIVE: 1 runs the network's 16->16 layers and its
                                    backward pass (training) on CUDA cores instead of
                                    tcgen05 (for comparison)                          */
    int32_t pcg_warm_start;      /* NATIVE: 1 (default) starts each step's Jacobi-PCG
                                    or multilevel FCG (pressure_method 0 or 2) from
                                    the previous step's pressure on the cells fluid in
                                    both; the stop test stays |r| <= tol |b|          */
    int32_t mg_coarse;           /* NATIVE, pressure_method 2: 0 (default) solves the
                                    coarsest level with the network, 1 with Jacobi
                                    sweeps only (the same V-cycle without the network),
                                    2 with Jacobi-PCG in one CTA (relative tolerance
                                    1e-3, at most 64 iterations; for comparison)       */
} flip_params;

/* Defaults for a mode (reference constants for FLIP_MODE_REFERENCE). */
void flip_default_params(int mode, flip_params* out);

/* Particles::Particles(uint size) (engine/particles.cu:15-40). */
int flip_create(uint64_t n, const flip_params* params, void* stream, flip_engine** out);
/* Particles::setDomain (engine/particles.cu:42-46).  NATIVE needs the voxel
 * counts 4*sizeX.. to be multiples of 8. */
int flip_set_domain(flip_engine* e, double nx, double ny, double nz, uint32_t x, uint32_t y, uint32_t z,
                    double cellSize);
/* Host upload / download of particle state (CudaVec::upload/download,
 * engine/cudaVec.cu:75-103).  The _f64 forms take the reference's double
 * arrays; the _f32 forms float arrays.  Velocities may be NULL. */
int flip_upload_particles_f64(flip_engine* e, const double* px, const double* py, const double* pz,
                              const double* vx, const double* vy, const double* vz, uint64_t n);
int flip_download_particles_f64(flip_engine* e, double* px, double* py, double* pz, double* vx, double* vy,
                                double* vz, uint64_t n);
int flip_upload_particles_f32(flip_engine* e, const float* px, const float* py, const float* pz,
                              const float* vx, const float* vy, const float* vz, uint64_t n);
int flip_download_particles_f32(flip_engine* e, float* px, float* py, float* pz, float* vx, float* vy, float* vz,
                                uint64_t n);
/* Optional static solid cells (NATIVE): mask of nx*ny*nz voxels, x fastest. */
int flip_set_solid_mask(flip_engine* e, const uint8_t* mask_host, uint64_t n_voxels);
/* NATIVE, no reference counterpart (the reference's solids are static, walls
 * only: particles.cu:479): the velocity of the interior solid cells.  Faces
 * between a solid and a non-solid cell carry it, so the pressure solve and the
 * projection see a moving obstacle; faces on the box walls stay 0. */
int flip_set_solid_velocity(flip_engine* e, double ux, double uy, double uz);

/* Per-stage methods of Particles (engine/particles.hu:17-43). */
int flip_align_particles_to_grid(flip_engine* e);   /* alignParticlesToGrid, particles.cu:48-50    */
int flip_sort_particles(flip_engine* e);            /* sortParticles, particles.cu:52-78           */
int flip_generate_voxels(flip_engine* e);           /* generateVoxels, particles.cu:323-368        */
int flip_particle_vel_to_voxels(flip_engine* e);    /* particleVelToVoxels, particles.cu:500-505   */
int flip_pressure_solve(flip_engine* e);            /* pressureSolve, particles.cu:507-555         */
int flip_update_voxel_velocities(flip_engine* e);   /* updateVoxelVelocities, particles.cu:557-560 */
int flip_voxel_vels_to_particles(flip_engine* e);   /* voxelVelsToParticles, particles.cu:742-749  */
int flip_advect_particles(flip_engine* e);          /* advectParticles, particles.cu:751-760       */
int flip_move_solid_particles(flip_engine* e);      /* moveSolidParticles, particles.cu:762-769    */
int flip_initialize(flip_engine* e);                /* initialize, particles.cu:805-812            */
int flip_solve_frame(flip_engine* e, double fps);   /* solveFrame, particles.cu:784-803            */
double flip_get_courant_dt(flip_engine* e);         /* getCourantDt, particles.cu:493-498          */
/* In native mode solveFrame takes sub-steps of min(max_substep_dt, the
 * Courant limit 0.7 h / max |v component|, the rest of the frame), with the
 * speed reduced on the device; flip_get_courant_dt returns that limit (0 at
 * rest).  With pressure_method 0 or 2 and stage timing off the whole frame is
 * one CUDA graph launch: a conditional loop over sub-steps whose dt the
 * device picks, each sub-step the graph of flip_step; the call synchronises
 * once, at the end of the frame. */
/* writePositionsToFile (particles.cu:817-828): "x, y, z" per line. */
int flip_write_positions_csv(flip_engine* e, const char* path);
/* Binary variant of the same frame (no reference counterpart): a 16-byte
 * header "FLIP2POS" + uint64 count (little endian), then count x 3 float32
 * (x, y, z interleaved).  FP32 positions at 12 B a particle instead of about
 * 30 B of text. */
int flip_write_positions_bin(flip_engine* e, const char* path);

/* One fixed-dt step of the whole path (bin, P2G, pressure, projection,
 * G2P + advection), asynchronous on the engine stream.  NATIVE with
 * pressure_method 0 or 2 and stage timing off: one CUDA graph launch (captured
 * on first use, with the solve's iteration loop and the Jacobi-PCG restart as
 * conditional nodes); the host reads nothing back -- flip_get_info and
 * flip_get_solve_info fetch the solve's outcome when called.  Otherwise the
 * stages are launched one by one and the pressure solve synchronises. */
int flip_step(flip_engine* e, double dt);
int flip_sync(flip_engine* e);
/* NATIVE, no reference counterpart: a host round trip per step.  Uploads
 * the particle state from the six host arrays (pinned memory lets the copies
 * run asynchronously), takes one step and downloads the new state into the
 * same arrays.  The copies run in 8 ranges on two copy streams; a range's
 * upload waits only for the previous call's download of that range, so one
 * call's download overlaps the next call's upload.  The call returns before
 * its download has finished: flip_sync (and every other engine call) waits
 * for it, and the host arrays must not be read or written before then. */
int flip_step_streamed_f32(flip_engine* e, float* px, float* py, float* pz, float* vx, float* vy, float* vz,
                           uint64_t n, double dt);

/* Buffers for inspection (device pointers lent, not transferred).  In
 * NATIVE mode FLIP_BUF_UX/UY/UZ are the face grids, FLIP_BUF_DIVU the
 * right-hand side b, FLIP_BUF_P the FP64 solution part and FLIP_BUF_RES the
 * solver's working residual: D^-1 r (r scaled by the inverse Jacobi diagonal)
 * after a Jacobi-PCG solve, r after a flexible one. */
typedef enum {
    FLIP_BUF_PX = 0, FLIP_BUF_PY, FLIP_BUF_PZ, FLIP_BUF_VX, FLIP_BUF_VY, FLIP_BUF_VZ,
    FLIP_BUF_KEYS, FLIP_BUF_PERM, FLIP_BUF_FLAGS, FLIP_BUF_STARTS, FLIP_BUF_YTABLE,
    FLIP_BUF_NODE_VOXELS, FLIP_BUF_VOXEL_IDS, FLIP_BUF_SOLIDS, FLIP_BUF_UX, FLIP_BUF_UY, FLIP_BUF_UZ,
    FLIP_BUF_DIVU, FLIP_BUF_P, FLIP_BUF_RES,
    /* NATIVE dense tile-blocked grids (slot = tile*512 + local voxel) */
    FLIP_BUF_GRID_U, FLIP_BUF_GRID_V, FLIP_BUF_GRID_W, FLIP_BUF_CELL_TYPE, FLIP_BUF_PRESSURE,
    FLIP_BUF_TILE_LIST,
    /* NATIVE grid velocity right after P2G (the FLIP "old" grid) */
    FLIP_BUF_GRID_U_P2G, FLIP_BUF_GRID_V_P2G, FLIP_BUF_GRID_W_P2G,
    /* NATIVE multilevel preconditioner, its coarsest level (tile-blocked on
     * that level's grid; empty until pressure_method 2 or flip_mg_* ran):
     * cell types, the last right-hand side and the last training error
     * sample of flip_mg_train_step */
    FLIP_BUF_MG_COARSE_TYPE, FLIP_BUF_MG_COARSE_R, FLIP_BUF_MG_COARSE_E,
    FLIP_BUF_COUNT
} flip_buffer;
/* elem_size: 1, 4 or 8 bytes; count: number of valid elements.
 * NATIVE FLIP_BUF_PRESSURE (FP64): the last solve's pressure on its fluid
 * cells, 0 elsewhere (the call first folds the solver's FP32 increments in). */
int flip_get_buffer(flip_engine* e, int which, void** dev_ptr, uint64_t* count, uint32_t* elem_size);
/* Copy a buffer of flip_get_buffer to host memory (bytes <= count*elem_size),
 * synchronising the engine stream; CudaVec::download (cudaVec.cu:80-86). */
int flip_read_buffer(flip_engine* e, int which, void* host_dst, uint64_t bytes);

/* ------------------------------------------------------------------ */
/* 3. Learned pressure preconditioner and standalone pressure problems  */
/*    (native-mode additions: no reference counterpart)                 */
/* ------------------------------------------------------------------ */
/* The network: 3^3 convolutions 3 -> 16 -> 16 -> 16 -> 1 channels with
 * dilations 1, 2, 4, 1, ReLU after the first three, no biases; inputs are
 * [r / rms(r), fluid flag, solid flag], the output is scaled by rms(r) and
 * kept on fluid cells.  BF16 weights and activations, FP32 accumulation.
 * Weights: FP32, layer after layer, each [27 taps][Cin][Cout]. */
uint64_t flip_lp_num_weights(void);
int flip_lp_init(flip_engine* e, uint64_t seed);                      /* He-normal init, Adam reset */
int flip_lp_set_weights(flip_engine* e, const float* w, uint64_t n);
int flip_lp_get_weights(flip_engine* e, float* w, uint64_t n);
int flip_lp_get_grad(flip_engine* e, float* g, uint64_t n);           /* last weight gradient       */

/* A pressure problem on the whole native grid (the learned-preconditioner
 * configuration): solid spheres, fluid below a surface, air above, and
 * b = -div(u) of Gaussian velocity impulses plus gravity. */
typedef struct {
    uint64_t seed;
    double surface_min, surface_max;   /* fluid surface height, fraction of ny        */
    double solid_fraction;             /* target solid volume fraction (0.10)         */
    double radius_min, radius_max;     /* sphere radii in voxels (4..16)              */
    int32_t impulses;                  /* Gaussian velocity impulses                  */
    int32_t reserved;
    double gravity_dt;                 /* gravity * dt added on fluid y faces         */
} flip_poisson_spec;
int flip_poisson_generate(flip_engine* e, const flip_poisson_spec* spec);
/* explicit problem: cell types (0 air, 1 fluid, 2 solid) and b, x fastest */
int flip_poisson_set(flip_engine* e, const uint8_t* type_lin, const float* b_lin);
typedef struct {
    int32_t iters;          /* iterations of the method asked for             */
    int32_t converged;      /* 1: true relative residual <= tol               */
    int32_t fell_back;      /* 1: FPCG missed its cap and Jacobi-PCG restarted */
    int32_t plain_iters;    /* iterations of that restart                     */
    double rel_residual;    /* FP64 true residual / |b|                       */
    double ms;              /* device time of the solve                       */
} flip_solve_info;
/* the last pressure solve: flip_poisson_solve's or a native step's (ms is
 * measured for a step only while stage timing is on).  After a native step
 * its pressure problem stays in place for flip_poisson_solve,
 * flip_lp_train_step and flip_lp_eval until the next step. */
int flip_get_solve_info(flip_engine* e, flip_solve_info* out);
/* method 0: Jacobi-PCG; 1: FPCG with the network preconditioner; 2: FPCG
 * with the multilevel preconditioner (flip_params.mg_coarse picks the
 * coarsest solve).  Methods 1 and 2 restart Jacobi-PCG from x = 0 when they
 * miss tol within max_iter or stall. */
int flip_poisson_solve(flip_engine* e, int method, double tol, int max_iter, flip_solve_info* info);
/* solution (FP64) in x-fastest order */
int flip_poisson_read_solution(flip_engine* e, double* x_lin);
/* The solver applies M(r) = N(r) + D^-1 r (network plus Jacobi).  One
 * training step on the current problem with a sample (r, e), A e = r:
 *   sample >= 0: x_k after `sample` Jacobi-PCG iterations from 0, r its
 *                residual and e = x* - x_k, x* the problem's converged
 *                solution (solved once per problem, or the solve just done);
 *   sample = -1: e white noise on the fluid cells and r = A e.
 * Loss L = |M(r) - e|_A^2 / |e|_A^2, one Adam step at rate lr; *loss is the
 * value before the step. */
int flip_lp_train_step(flip_engine* e, int sample, float lr, double* loss);
/* evaluate on a given r and e (x fastest) of the current problem: z = N(r)
 * out (x fastest, may be NULL), the loss, and with want_grad the weight
 * gradient (flip_lp_get_grad) without updating the weights */
int flip_lp_eval(flip_engine* e, const float* r_lin, const float* e_lin, float* z_lin, double* loss, int want_grad);

/* Multilevel preconditioner (pressure_method 2).  No reference counterpart.
 * The network's weights are the ones above; here they act on the coarsest
 * level of the V-cycle.
 * One V-cycle z = M(r) on the current problem, r and z x fastest (for
 * checks against a CPU restatement). */
int flip_mg_apply(flip_engine* e, const float* r_lin, float* z_lin);
/* one training step of the network as the coarsest solve: sample k >= 0
 * takes the coarsest right-hand side that a V-cycle makes of the residual
 * after k Jacobi-PCG iterations on the current problem, with its coarse
 * solution from CG; sample -1 a white-noise coarse error e and r = A e.
 * Loss as flip_lp_train_step's (A-norm error of N(r) + D^-1 r on the
 * coarsest level); lr = 0 computes loss and gradient without a step. */
int flip_mg_train_step(flip_engine* e, int sample, float lr, double* loss);

typedef struct {
    uint32_t nodes;          /* occupied root cells (REFERENCE) / tiles (NATIVE)   */
    uint32_t voxels;         /* used voxels (REFERENCE) / grid tiles (NATIVE)      */
    int32_t pressure_iters;  /* last solve                                        */
    int32_t converged;       /* 1 if the last solve met its tolerance             */
    double dt;               /* last dt                                           */
    double residual;         /* last terminating residual (relative for NATIVE)  */
    double elapsed_time;
    uint64_t n;
    uint32_t error_flags;    /* device error bits seen since setDomain (bit 0: a
                                look-back wait of a sort or scan timed out, which
                                the next synchronising call -- flip_sync,
                                flip_solve_frame, generateVoxels, the end of each
                                native pressure solve -- also returns as
                                FLIP_ERR_TIMEOUT; bit 2: a tensor-core wait of the
                                learned preconditioner timed out)                */
    uint32_t launches;       /* kernels this engine launched since creation      */
    uint64_t solves;         /* NATIVE: pressure solves since setDomain           */
    uint64_t fallbacks;      /* NATIVE: of those, flexible solves that missed tol
                                and restarted Jacobi-PCG                          */
    uint64_t pressure_iters_total; /* NATIVE: their iterations, restarts included */
    uint64_t graph_steps;    /* NATIVE: steps that ran as CUDA graph launches     */
} flip_info;
int flip_get_info(flip_engine* e, flip_info* out);
/* Per-stage device times of flip_step (CUDA events on the engine stream).
 * With timing enabled every step synchronises at its end and adds its stage
 * times to the running totals; flip_get_stage_ms returns the totals (ms) of
 * FLIP_NUM_STAGES stages: keys, sort, gather, segment heads, grid clear, P2G,
 * tile dilation, normalise+gravity, PCG setup, PCG iterations, projection,
 * G2P+advection; and resets them when reset != 0. */
#define FLIP_NUM_STAGES 12
int flip_set_timing(flip_engine* e, int enable);
int flip_get_stage_ms(flip_engine* e, double* ms, int n, int reset);
const char* flip_last_error(flip_engine* e);
int flip_destroy(flip_engine* e);

#ifdef __cplusplus
}
#endif
#endif /* FLIP2_B200_H */
