// ref_harness.cu -- drives the reference engine (built from its own sources
// by oracle/Makefile into oracle/_ref/) stage by stage on seeded inputs and
// hands every intermediate buffer back to Python (tests/golden/make_golden.py)
// through a small C API.  TEST INFRASTRUCTURE ONLY: it produces the golden
// fixtures that pin the CPU oracle; nothing in the product links it.
//
// It uses the hook the reference provides for this purpose: Particles
// declares `friend class ParticleSystemTester` (engine/particles.hu:94).
// This file defines its own ParticleSystemTester (engine/testing.h is not
// included) to read and write the private CudaVec buffers.
//
// Only stages whose device code was checked to stay in bounds on inputs
// strictly inside the box with sizeX == sizeZ are exposed; moveSolids
// (engine/particles.cu:674-740) is not, because its search loop can index
// past its shared-memory list when a node has no solid voxel.
#include "particles.hu"
#include "algorithms/voxelSolveFunctions.hu"
#include <cstdio>
#include <cstring>
#include <vector>
#include <cstdint>

// Kernels defined in the reference's translation units, launched here
// directly so the P2G weight-sum scratch can be cleared between axes.
__global__ void gatherParticleVelsToVoxels(uint numUsedGridNodes, uint numParticles, uint numVoxelsPerNode,
    uint numVoxels1D, uint* gridNodeIndicesToFirstParticleIndex, uint* gridPosition, double* px, double* py,
    double* pz, double* vDim, uint* numVoxelsEachNode, uint* voxelIDs, double* voxelUs, char* solids,
    double radius, Grid grid, uint refinementLevel, VelocityGatherDimension dimension);
__global__ void GSiteration(uint numVoxelsPerNode, uint numVoxels1D, uint refinementLevel, double radius,
    const uint* nodeIndexUsedVoxels, const uint* voxelIDs, const char* solids, const double* divU, double* p,
    double* residuals, double density, double dt, Grid grid, bool red, double w);

// Zero the whole shared-memory window of every SM, so that kernels launched
// next start from zeroed shared memory (gatherParticleVelsToVoxels reads its
// weight sums before writing them, engine/particles.cu:408-415).
__global__ void harness_scrub_smem(int words) {
    extern __shared__ uint4 s[];
    for (int i = threadIdx.x; i < words; i += blockDim.x) s[i] = make_uint4(0, 0, 0, 0);
}

class ParticleSystemTester {
public:
    explicit ParticleSystemTester(uint n) : p(n) {}
    Particles p;
    double lastDt = 0.0;

    static int create(uint32_t n, double nx, double ny, double nz, uint32_t X, uint32_t Y, uint32_t Z, double cell, void** out);
    static int upload(void* h, const double* px, const double* py, const double* pz,
                      const double* vx, const double* vy, const double* vz);
    static int set_time(void* h, double frameDt, double elapsedThisFrame);
    static int stage(void* h, int stage, double dt_arg);
    static int info(void* h, uint32_t* nodes, uint32_t* voxels, double* dt);
    static int download(void* h, int buf, void* dst, size_t cap_bytes, size_t* out_bytes);
    static int upload_buf(void* h, int buf, const void* src, size_t bytes);
};


enum {
    BUF_PX = 0, BUF_PY, BUF_PZ, BUF_VX, BUF_VY, BUF_VZ,
    BUF_KEYS, BUF_PERM, BUF_FLAGS, BUF_STARTS, BUF_YTABLE,
    BUF_NODE_VOXELS, BUF_VOXEL_IDS, BUF_SOLIDS, BUF_UX, BUF_UY, BUF_UZ,
    BUF_DIVU, BUF_P, BUF_RES
};

static void scrub() {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, dev);
    int bytes = (int)prop.sharedMemPerBlockOptin;
    cudaFuncSetAttribute(harness_scrub_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    harness_scrub_smem<<<prop.multiProcessorCount * 4, 1024, bytes>>>(bytes / 16);
    cudaDeviceSynchronize();
}

template <typename T>
static int copy_out(CudaVec<T>& v, void* dst, size_t cap_bytes, size_t* out_bytes) {
    size_t b = sizeof(T) * (size_t)v.size();
    *out_bytes = b;
    if (!dst) return 0;
    if (b > cap_bytes) return -2;
    return cudaMemcpy(dst, v.devPtr(), b, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -1;
}


int ParticleSystemTester::create(uint32_t n, double nx, double ny, double nz, uint32_t X, uint32_t Y, uint32_t Z, double cell, void** out) {
    ParticleSystemTester* t = new ParticleSystemTester(n);
    t->p.setDomain(nx, ny, nz, X, Y, Z, cell);
    t->p.elapsedTime = 0.0;
    t->p.elapsedTimeThisFrame = 0.0;
    t->p.frameDt = 1.0 / 24.0;
    t->p.dt = t->p.frameDt / 10.0;
    cudaStreamSynchronize(t->p.stream);
    *out = t;
    return 0;
}

int ParticleSystemTester::upload(void* h, const double* px, const double* py, const double* pz,
               const double* vx, const double* vy, const double* vz) {
    Particles& p = ((ParticleSystemTester*)h)->p;
    size_t b = sizeof(double) * p.size;
    const double* src[6] = {px, py, pz, vx, vy, vz};
    CudaVec<double>* dst[6] = {&p.px, &p.py, &p.pz, &p.vx, &p.vy, &p.vz};
    for (int i = 0; i < 6; ++i)
        if (cudaMemcpy(dst[i]->devPtr(), src[i], b, cudaMemcpyHostToDevice) != cudaSuccess) return -1;
    return 0;
}

int ParticleSystemTester::set_time(void* h, double frameDt, double elapsedThisFrame) {
    Particles& p = ((ParticleSystemTester*)h)->p;
    p.frameDt = frameDt;
    p.elapsedTimeThisFrame = elapsedThisFrame;
    return 0;
}

// stage ids
//  0 alignParticlesToGrid      1 sortParticles          2 generateVoxels
//  3 P2G (3 axes, shared memory cleared before each axis launch)
//  4 particleVelToVoxels as shipped (no clearing)
//  5 applyGravity(dt_arg) + cudaCalcDivU
//  6 pressureSolve             7 updateVoxelVelocities  8 voxelVelsToParticles
//  9 advectParticles          10 one red + one black GSiteration launch with dt_arg
int ParticleSystemTester::stage(void* h, int stage, double dt_arg) {
    ParticleSystemTester* t = (ParticleSystemTester*)h;
    Particles& p = t->p;
    switch (stage) {
    case 0: p.alignParticlesToGrid(); break;
    case 1: p.sortParticles(); break;
    case 2: p.generateVoxels(); break;
    case 3: {
        CudaVec<double>* v[3] = {&p.vx, &p.vy, &p.vz};
        CudaVec<double>* u[3] = {&p.voxelsUx, &p.voxelsUy, &p.voxelsUz};
        VelocityGatherDimension d[3] = {VelocityGatherDimension::X, VelocityGatherDimension::Y, VelocityGatherDimension::Z};
        for (int a = 0; a < 3; ++a) {
            scrub();
            gatherParticleVelsToVoxels<<<p.numUsedGridNodes, 32, 2 * sizeof(double) * p.numVoxelsPerNode + p.numVoxelsPerNode, p.stream>>>(
                p.numUsedGridNodes, p.size, p.numVoxelsPerNode, p.numVoxels1D, p.gridNodeIndicesToFirstParticleIndex.devPtr(),
                p.gridCell.devPtr(), p.px.devPtr(), p.py.devPtr(), p.pz.devPtr(), v[a]->devPtr(), p.nodeIndexUsedVoxels.devPtr(),
                p.voxelIDsUsed.devPtr(), u[a]->devPtr(), p.solids.devPtr(), p.radius, p.grid, p.refinementLevel, d[a]);
            cudaStreamSynchronize(p.stream);
        }
        break;
    }
    case 4: p.particleVelToVoxels(); break;
    case 5:
        p.dt = dt_arg;
        applyGravity(p.solids, p.voxelsUy, dt_arg, p.stream);
        cudaCalcDivU(p.nodeIndexUsedVoxels, p.voxelIDsUsed, p.voxelsUx, p.voxelsUy, p.voxelsUz, p.radius, p.refinementLevel,
                     p.grid, p.yDimNumUsedGridNodes, p.gridNodeIndicesToFirstParticleIndex, p.gridCell, p.numVoxelsPerNode,
                     p.numVoxels1D, p.divU, p.stream);
        break;
    case 6: p.pressureSolve(); t->lastDt = p.dt; break;
    case 7: p.updateVoxelVelocities(); break;
    case 8: p.voxelVelsToParticles(); break;
    case 9: p.advectParticles(); break;
    case 10:
        for (int red = 1; red >= 0; --red) {
            GSiteration<<<p.nodeIndexUsedVoxels.size(), 256, (3 * sizeof(double) + sizeof(uint) + sizeof(char)) * p.numVoxelsPerNode, p.stream>>>(
                p.numVoxelsPerNode, p.numVoxels1D, p.refinementLevel, p.radius, p.nodeIndexUsedVoxels.devPtr(), p.voxelIDsUsed.devPtr(),
                p.solids.devPtr(), p.divU.devPtr(), p.p.devPtr(), p.residuals.devPtr(), 0.014, dt_arg, p.grid, red == 1, 1.9);
        }
        break;
    default: return -3;
    }
    cudaError_t e = cudaStreamSynchronize(p.stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    return e == cudaSuccess ? 0 : -(int)e - 100;
}

int ParticleSystemTester::info(void* h, uint32_t* nodes, uint32_t* voxels, double* dt) {
    ParticleSystemTester* t = (ParticleSystemTester*)h;
    *nodes = t->p.numUsedGridNodes;
    *voxels = t->p.voxelIDsUsed.size();
    *dt = t->p.dt;
    return 0;
}

int ParticleSystemTester::download(void* h, int buf, void* dst, size_t cap_bytes, size_t* out_bytes) {
    Particles& p = ((ParticleSystemTester*)h)->p;
    switch (buf) {
    case BUF_PX: return copy_out(p.px, dst, cap_bytes, out_bytes);
    case BUF_PY: return copy_out(p.py, dst, cap_bytes, out_bytes);
    case BUF_PZ: return copy_out(p.pz, dst, cap_bytes, out_bytes);
    case BUF_VX: return copy_out(p.vx, dst, cap_bytes, out_bytes);
    case BUF_VY: return copy_out(p.vy, dst, cap_bytes, out_bytes);
    case BUF_VZ: return copy_out(p.vz, dst, cap_bytes, out_bytes);
    case BUF_KEYS: return copy_out(p.gridCell, dst, cap_bytes, out_bytes);
    case BUF_PERM: return copy_out(p.reorderedGridIndices, dst, cap_bytes, out_bytes);
    case BUF_FLAGS: return copy_out(p.uniqueGridNodeIndices, dst, cap_bytes, out_bytes);
    case BUF_STARTS: return copy_out(p.gridNodeIndicesToFirstParticleIndex, dst, cap_bytes, out_bytes);
    case BUF_YTABLE: return copy_out(p.yDimNumUsedGridNodes, dst, cap_bytes, out_bytes);
    case BUF_NODE_VOXELS: return copy_out(p.nodeIndexUsedVoxels, dst, cap_bytes, out_bytes);
    case BUF_VOXEL_IDS: return copy_out(p.voxelIDsUsed, dst, cap_bytes, out_bytes);
    case BUF_SOLIDS: return copy_out(p.solids, dst, cap_bytes, out_bytes);
    case BUF_UX: return copy_out(p.voxelsUx, dst, cap_bytes, out_bytes);
    case BUF_UY: return copy_out(p.voxelsUy, dst, cap_bytes, out_bytes);
    case BUF_UZ: return copy_out(p.voxelsUz, dst, cap_bytes, out_bytes);
    case BUF_DIVU: return copy_out(p.divU, dst, cap_bytes, out_bytes);
    case BUF_P: return copy_out(p.p, dst, cap_bytes, out_bytes);
    case BUF_RES: return copy_out(p.residuals, dst, cap_bytes, out_bytes);
    default: return -3;
    }
}

// Upload into an existing device buffer of matching size (used to feed a
// stage the exact inputs of the oracle, e.g. voxel velocities before G2P).
int ParticleSystemTester::upload_buf(void* h, int buf, const void* src, size_t bytes) {
    Particles& p = ((ParticleSystemTester*)h)->p;
    void* d = nullptr;
    size_t have = 0;
    switch (buf) {
    case BUF_UX: d = p.voxelsUx.devPtr(); have = 8 * (size_t)p.voxelsUx.size(); break;
    case BUF_UY: d = p.voxelsUy.devPtr(); have = 8 * (size_t)p.voxelsUy.size(); break;
    case BUF_UZ: d = p.voxelsUz.devPtr(); have = 8 * (size_t)p.voxelsUz.size(); break;
    case BUF_P: d = p.p.devPtr(); have = 8 * (size_t)p.p.size(); break;
    case BUF_DIVU: d = p.divU.devPtr(); have = 8 * (size_t)p.divU.size(); break;
    default: return -3;
    }
    if (bytes != have) return -2;
    return cudaMemcpy(d, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : -1;
}



extern "C" {
int ref_create(uint32_t n, double nx, double ny, double nz, uint32_t X, uint32_t Y, uint32_t Z, double cell, void** out) {
    return ParticleSystemTester::create(n, nx, ny, nz, X, Y, Z, cell, out);
}
int ref_upload(void* h, const double* px, const double* py, const double* pz, const double* vx, const double* vy, const double* vz) {
    return ParticleSystemTester::upload(h, px, py, pz, vx, vy, vz);
}
int ref_set_time(void* h, double frameDt, double elapsedThisFrame) { return ParticleSystemTester::set_time(h, frameDt, elapsedThisFrame); }
int ref_stage(void* h, int stage, double dt_arg) { return ParticleSystemTester::stage(h, stage, dt_arg); }
int ref_info(void* h, uint32_t* nodes, uint32_t* voxels, double* dt) { return ParticleSystemTester::info(h, nodes, voxels, dt); }
int ref_download(void* h, int buf, void* dst, size_t cap_bytes, size_t* out_bytes) {
    return ParticleSystemTester::download(h, buf, dst, cap_bytes, out_bytes);
}
int ref_upload_buf(void* h, int buf, const void* src, size_t bytes) { return ParticleSystemTester::upload_buf(h, buf, src, bytes); }
void ref_destroy(void* h) { delete (ParticleSystemTester*)h; }
}  // extern "C"
