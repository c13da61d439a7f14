// ref_kernels.cuh -- launchers of the reference-math kernels (ref_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "flip2_b200.h"

namespace flip {

int ref_launch_keys(double* px, double* py, double* pz, uint64_t n, const flip_grid& g, uint32_t* keys, uint32_t* idx,
                    cudaStream_t s);
int ref_launch_ydim(const uint32_t* starts, const uint32_t* keys, uint32_t nodes, const flip_grid& g, uint32_t* table,
                    cudaStream_t s);
int ref_launch_voxel_counts(const uint32_t* starts, const uint32_t* keys, uint32_t nodes, uint64_t n, const double* px,
                            const double* py, const double* pz, const flip_grid& g, uint32_t* counts, uint32_t* masks,
                            cudaStream_t s);
int ref_launch_voxel_ids(const uint32_t* keys, uint32_t nodes, const uint32_t* masks, const uint32_t* node_voxels,
                         const flip_grid& g, uint32_t* voxel_ids, int8_t* solids, cudaStream_t s);
int ref_launch_p2g(const uint32_t* starts, const uint32_t* keys, uint32_t nodes, uint64_t n, const double* px,
                   const double* py, const double* pz, const double* vx, const double* vy, const double* vz,
                   const uint32_t* node_voxels, const uint32_t* voxel_ids, const int8_t* solids, const flip_grid& g,
                   double* ux, double* uy, double* uz, cudaStream_t s);
int ref_launch_g2p(const uint32_t* starts, const uint32_t* keys, uint32_t nodes, uint64_t n, const double* px,
                   const double* py, const double* pz, const uint32_t* node_voxels, const uint32_t* voxel_ids,
                   const double* ux, const double* uy, const double* uz, const flip_grid& g, double* vx, double* vy,
                   double* vz, cudaStream_t s);
int ref_launch_advect(uint64_t n, double dt, double* px, double* py, double* pz, const double* vx, const double* vy,
                      const double* vz, cudaStream_t s);
int ref_launch_gravity(uint64_t nvox, const int8_t* solids, double* uy, double dt, int remove, cudaStream_t s);
int ref_launch_divergence(uint32_t nodes, const uint32_t* node_voxels, const uint32_t* voxel_ids, const double* ux,
                          const double* uy, const double* uz, const flip_grid& g, const uint32_t* ytable,
                          const uint32_t* starts, const uint32_t* keys, double* divU, cudaStream_t s);
int ref_launch_gs(uint32_t nodes, const uint32_t* node_voxels, const uint32_t* voxel_ids, const int8_t* solids,
                  const double* divU, double* p, double* res, double scale, double w, uint32_t iters, cudaStream_t s);
int ref_launch_velocity_update(uint32_t nodes, const uint32_t* node_voxels, const uint32_t* voxel_ids,
                               const int8_t* solids, const double* p, double* ux, double* uy, double* uz, double scale,
                               cudaStream_t s);
int ref_launch_getmax_level(uint64_t n, const double* a, double* out, int absolute, cudaStream_t s);
int ref_launch_move_solids(uint32_t nodes, uint64_t n, const uint32_t* starts, const uint32_t* keys, double* px,
                           double* py, double* pz, const uint32_t* node_voxels, const uint32_t* voxel_ids,
                           const int8_t* solids, const flip_grid& g, cudaStream_t s);

int ref_gather_f64(const uint32_t* perm, uint64_t n, const double* in, double* out, cudaStream_t s);

// scan.cu
int launch_scan(int mode, const uint32_t* in, uint32_t* out, uint64_t n, void* scratch, size_t bytes, cudaStream_t s,
                uint32_t* starts, uint32_t* node_keys, uint32_t* d_count, uint32_t* err_accum, uint32_t spin_limit,
                uint32_t tile_base);
size_t scan_scratch_bytes(uint64_t n);

}  // namespace flip
