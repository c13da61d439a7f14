// particles.hpp -- C++ facade with the reference engine's class names over the
// flip2_b200 C ABI, so that drivers written against engine/particles.hu,
// engine/cudaVec.hu and engine/grid.hpp (engine/main.cu, engine/testing.h)
// compile against this library with a changed include path.
//
//   Grid      engine/grid.hpp:8-38        (header-only, same fields)
//   CudaVec   engine/cudaVec.hu:17-53     (owning device buffer + host mirror)
//   Particles engine/particles.hu:11-95   (methods forward to flip_* calls)
//
// Differences a caller can see: errors throw flip2::Error instead of exiting
// the process (the reference's gpuErrchk calls exit(), typedefs.h:12-20), and
// state can be read through download() instead of a friend class.
#pragma once
#include <cuda_runtime.h>
#include <stdexcept>
#include <string>
#include <vector>
#include "../flip2_b200.h"

namespace flip2 {

typedef unsigned int uint;

class Error : public std::runtime_error {
public:
    Error(int status, const std::string& what) : std::runtime_error(what), status(status) {}
    int status;
};

inline void check(int rc, const char* what, flip_engine* e = nullptr) {
    if (rc != FLIP_OK) {
        std::string msg = std::string(what) + ": " + flip_status_string(rc);
        const char* d = flip_last_error(e);
        if (d && *d) msg += std::string(" (") + d + ")";
        throw Error(rc, msg);
    }
}
inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(FLIP_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------- Grid
class Grid {
public:
    Grid(float nx = 0.0f, float ny = 0.0f, float nz = 0.0f, uint numGridsX = 0, uint numGridsY = 0, uint numGridsZ = 0,
         float gridSize = 0.0f)
        : negX(nx), negY(ny), negZ(nz), sizeX(numGridsX), sizeY(numGridsY), sizeZ(numGridsZ), cellSize(gridSize) {}
    void setNegativeCorner(float nx, float ny, float nz) { negX = nx; negY = ny; negZ = nz; }
    void setSize(uint x, uint y, uint z, float gridSize) { cellSize = gridSize; sizeX = x; sizeY = y; sizeZ = z; }
    flip_grid c() const { return flip_grid{negX, negY, negZ, sizeX, sizeY, sizeZ, cellSize}; }
    float negX, negY, negZ;
    uint sizeX, sizeY, sizeZ;
    float cellSize;
};

// ------------------------------------------------------------- CudaVec
template <typename T>
class CudaVec {
public:
    CudaVec() = default;
    explicit CudaVec(const uint& size) { resize(size); }
    CudaVec(const CudaVec&) = delete;
    CudaVec& operator=(const CudaVec&) = delete;
    ~CudaVec() { clear(); }

    void resize(const uint& size) {
        release();
        numElements = size;
        vec.resize(size);
        if (size) cuda_check(cudaMalloc((void**)&d_vec, sizeof(T) * size), "cudaMalloc");
    }
    void resizeAsync(const uint& size, const cudaStream_t& stream) {
        release(stream);
        numElements = size;
        if (size) cuda_check(cudaMallocAsync((void**)&d_vec, sizeof(T) * size, stream), "cudaMallocAsync");
    }
    T& operator[](const uint& i) { return vec[i]; }
    const T& operator[](const uint& i) const { return vec[i]; }
    void upload() { upload(nullptr); cuda_check(cudaDeviceSynchronize(), "cudaDeviceSynchronize"); }
    void upload(cudaStream_t stream) {
        if (vec.size() != numElements) throw Error(FLIP_ERR_ARG, "CudaVec::upload: host and device sizes differ");
        cuda_check(cudaMemcpyAsync(d_vec, vec.data(), sizeof(T) * numElements, cudaMemcpyHostToDevice, stream), "upload");
    }
    void download() { download(nullptr); cuda_check(cudaDeviceSynchronize(), "cudaDeviceSynchronize"); }
    void download(cudaStream_t stream) {
        if (vec.size() != numElements) vec.resize(numElements);
        cuda_check(cudaMemcpyAsync(vec.data(), d_vec, sizeof(T) * numElements, cudaMemcpyDeviceToHost, stream), "download");
    }
    // adopt a device pointer; the previous buffer is freed (cudaVec.cu:133-149)
    void swapDevicePtr(T* p) {
        if (d_vec && d_vec != p) cudaFree(d_vec);
        d_vec = p;
    }
    void swapDevicePtrAsync(T* p, cudaStream_t stream) {
        if (d_vec && d_vec != p) cudaFreeAsync(d_vec, stream);
        d_vec = p;
    }
    T* devPtr() { return d_vec; }
    const T* devPtr() const { return d_vec; }
    void clear() { release(); vec.clear(); numElements = 0; }
    void clearAsync(cudaStream_t stream) { release(stream); vec.clear(); numElements = 0; }
    void zeroDevice() { zeroDeviceAsync(nullptr); }
    void zeroDeviceAsync(cudaStream_t stream) {
        if (numElements) cuda_check(cudaMemsetAsync(d_vec, 0, sizeof(T) * numElements, stream), "cudaMemsetAsync");
    }
    // the reference's getMax, implemented for double (the only type it calls it on)
    T getMax(cudaStream_t stream, bool abs = false);
    uint size() const { return numElements; }

private:
    void release(cudaStream_t stream = nullptr) {
        if (d_vec) {
            if (stream) cudaFreeAsync(d_vec, stream);
            else cudaFree(d_vec);
        }
        d_vec = nullptr;
    }
    std::vector<T> vec;
    T* d_vec = nullptr;
    uint numElements = 0;
};

template <>
inline double CudaVec<double>::getMax(cudaStream_t stream, bool abs) {
    size_t nb = flip_ref_getmax_scratch_bytes(numElements);
    void* scratch = nullptr;
    cuda_check(cudaMallocAsync(&scratch, nb, stream), "cudaMallocAsync");
    double out = 0.0;
    int rc = flip_ref_getmax_f64(d_vec, numElements, abs ? 1 : 0, scratch, nb, &out, stream);
    cudaFreeAsync(scratch, stream);
    check(rc, "CudaVec::getMax");
    return out;
}

// ----------------------------------------------------------- Particles
class Particles {
public:
    explicit Particles(uint size, int mode = FLIP_MODE_REFERENCE, cudaStream_t stream = nullptr) : size(size) {
        flip_params p;
        flip_default_params(mode, &p);
        check(flip_create(size, &p, (void*)stream, &e), "flip_create");
    }
    Particles(uint size, const flip_params& p, cudaStream_t stream = nullptr) : size(size) {
        check(flip_create(size, &p, (void*)stream, &e), "flip_create");
    }
    Particles(const Particles&) = delete;
    Particles& operator=(const Particles&) = delete;
    ~Particles() { flip_destroy(e); }

    void setDomain(double nx, double ny, double nz, uint x, uint y, uint z, double cellSize) {
        check(flip_set_domain(e, nx, ny, nz, x, y, z, cellSize), "setDomain", e);
        grid = Grid((float)nx, (float)ny, (float)nz, x, y, z, (float)cellSize);
    }
    void alignParticlesToGrid() { check(flip_align_particles_to_grid(e), "alignParticlesToGrid", e); }
    void sortParticles() { check(flip_sort_particles(e), "sortParticles", e); }
    void generateVoxels() { check(flip_generate_voxels(e), "generateVoxels", e); }
    void particleVelToVoxels() { check(flip_particle_vel_to_voxels(e), "particleVelToVoxels", e); }
    void setupCudaDevices() {}
    void pressureSolve() { check(flip_pressure_solve(e), "pressureSolve", e); }
    void updateVoxelVelocities() { check(flip_update_voxel_velocities(e), "updateVoxelVelocities", e); }
    void advectParticles() { check(flip_advect_particles(e), "advectParticles", e); }
    void solveFrame(double fps) { check(flip_solve_frame(e, fps), "solveFrame", e); }
    void initialize() { check(flip_initialize(e), "initialize", e); }
    void voxelVelsToParticles() { check(flip_voxel_vels_to_particles(e), "voxelVelsToParticles", e); }
    void moveSolidParticles() { check(flip_move_solid_particles(e), "moveSolidParticles", e); }
    void writePositionsToBinaryFile(const std::string& fileName) {
        check(flip_write_positions_bin(e, fileName.c_str()), "writePositionsToBinaryFile", e);
    }
    void writePositionsToFile(const std::string& fileName) {
        check(flip_write_positions_csv(e, fileName.c_str()), "writePositionsToFile", e);
    }
    double getCourantDt() { return flip_get_courant_dt(e); }

    // host access in place of the friend class
    void upload(const std::vector<double>& px, const std::vector<double>& py, const std::vector<double>& pz,
                const std::vector<double>* vx = nullptr, const std::vector<double>* vy = nullptr,
                const std::vector<double>* vz = nullptr) {
        check(flip_upload_particles_f64(e, px.data(), py.data(), pz.data(), vx ? vx->data() : nullptr,
                                        vy ? vy->data() : nullptr, vz ? vz->data() : nullptr, size),
              "upload", e);
    }
    void download(std::vector<double>& px, std::vector<double>& py, std::vector<double>& pz) {
        px.resize(size); py.resize(size); pz.resize(size);
        check(flip_download_particles_f64(e, px.data(), py.data(), pz.data(), nullptr, nullptr, nullptr, size),
              "download", e);
    }
    flip_info info() {
        flip_info i;
        check(flip_get_info(e, &i), "info", e);
        return i;
    }
    flip_engine* handle() { return e; }

    uint size;
    Grid grid;

private:
    flip_engine* e = nullptr;
};

}  // namespace flip2
