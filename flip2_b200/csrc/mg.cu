// mg.cu -- V-cycle kernels of the multilevel learned preconditioner (mg.cuh).
//
// Every level is tile-blocked like the solver's grid (slot = tile * 512 +
// (i & 7) + 8 (j & 7) + 64 (k & 7)).  The smoothing kernels walk a tile list
// with one CTA of 512 threads per tile and one thread per cell; neighbours
// come from global memory (the coarse levels are small enough to stay in L2).
// Non-fluid cells carry 0 in every vector, so the 7-point operator needs only
// the fluid bit and the non-solid neighbour count of the PCG cell code.
#include "common.cuh"
#include "mg.cuh"

namespace flip {

__device__ __forceinline__ uint32_t mg_slot(int i, int j, int k, const NatDims& D) {
    uint32_t t = (uint32_t)((i >> 3) + D.tx * ((j >> 3) + D.ty * (k >> 3)));
    return (t << 9) | (uint32_t)((i & 7) | ((j & 7) << 3) | ((k & 7) << 6));
}
__device__ __forceinline__ void mg_cell_of(uint32_t key, int tid, const NatDims& D, int& i, int& j, int& k) {
    i = 8 * (int)(key % D.tx) + (tid & 7);
    j = 8 * (int)((key / D.tx) % D.ty) + ((tid >> 3) & 7);
    k = 8 * (int)(key / (D.tx * D.ty)) + (tid >> 6);
}
__device__ __forceinline__ bool mg_in(int i, int j, int k, const NatDims& D) {
    return i >= 0 && j >= 0 && k >= 0 && i < D.nx && j < D.ny && k < D.nz;
}
__device__ __forceinline__ float mg_dinv(uint8_t c) {
    const uint32_t d = c & 7u;
    return d ? 1.0f / (float)d : 0.0f;
}
// sum over the fluid neighbours of (i, j, k) of val(slot)
template <class F>
__device__ __forceinline__ float mg_nb_sum(int i, int j, int k, const NatDims& D, const uint8_t* __restrict__ cell, F val) {
    const int oi[6] = {-1, 1, 0, 0, 0, 0}, oj[6] = {0, 0, -1, 1, 0, 0}, ok[6] = {0, 0, 0, 0, -1, 1};
    float s = 0.0f;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const int a = i + oi[q], b = j + oj[q], c = k + ok[q];
        if (!mg_in(a, b, c, D)) continue;
        const uint32_t u = mg_slot(a, b, c, D);
        if (cell[u] & kCellFluid) s += val(u);
    }
    return s;
}
__device__ __forceinline__ bool mg_halted(const int* halt) { return halt && *halt; }

// ------------------------------------------------------------ hierarchy
// coarse type from the 8 children: air if any child is air, else fluid if any
// is fluid, else solid; cells past the level's extent are solid
__global__ void __launch_bounds__(512) mg_coarsen_kernel(MgLevel F, MgLevel C, const int* halt) {
    if (mg_halted(halt)) return;
    const uint32_t n = C.ntiles * 512u;
    for (uint32_t s = blockIdx.x * 512u + threadIdx.x; s < n; s += gridDim.x * 512u) {
        int I, J, K;
        mg_cell_of(s >> 9, (int)(s & 511u), C.D, I, J, K);
        uint8_t t = kSolid;
        if (I < C.ex && J < C.ey && K < C.ez) {
            bool air = false, fluid = false;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int i = 2 * I + (c & 1), j = 2 * J + ((c >> 1) & 1), k = 2 * K + (c >> 2);
                if (i >= F.ex || j >= F.ey || k >= F.ez) continue;  // solid
                const uint8_t ft = F.type[mg_slot(i, j, k, F.D)];
                air |= ft == kAir;
                fluid |= ft == kFluid;
            }
            t = air ? kAir : (fluid ? kFluid : kSolid);
        }
        C.type[s] = t;
    }
}
// PCG cell codes of a coarse level: fluid bit and the non-solid neighbour count
__global__ void __launch_bounds__(512) mg_codes_kernel(MgLevel C, const int* halt) {
    if (mg_halted(halt)) return;
    const uint32_t n = C.ntiles * 512u;
    const int oi[6] = {-1, 1, 0, 0, 0, 0}, oj[6] = {0, 0, -1, 1, 0, 0}, ok[6] = {0, 0, 0, 0, -1, 1};
    for (uint32_t s = blockIdx.x * 512u + threadIdx.x; s < n; s += gridDim.x * 512u) {
        uint8_t code = 0;
        if (C.type[s] == kFluid) {
            int i, j, k;
            mg_cell_of(s >> 9, (int)(s & 511u), C.D, i, j, k);
            uint32_t d = 0;
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                const int a = i + oi[q], b = j + oj[q], c = k + ok[q];
                if (mg_in(a, b, c, C.D) && C.type[mg_slot(a, b, c, C.D)] != kSolid) ++d;
            }
            code = (uint8_t)(kCellFluid | d);
        }
        C.cell[s] = code;
    }
}

// ------------------------------------------------------------ smoothing
// pre-smoothing from zero: t1 = w D^-1 r, t = t1 + w D^-1 (r - A t1)
__global__ void __launch_bounds__(512) mg_pre_kernel(MgLevel L, const int* halt) {
    if (mg_halted(halt)) return;
    const uint32_t n = *L.d_ntiles;
    for (uint32_t tt = blockIdx.x; tt < n; tt += gridDim.x) {
        const uint32_t key = L.tiles[tt];
        const uint32_t s = (key << 9) | threadIdx.x;
        const uint8_t c = L.cell[s];
        float out = 0.0f;
        if (c & kCellFluid) {
            int i, j, k;
            mg_cell_of(key, threadIdx.x, L.D, i, j, k);
            const float di = mg_dinv(c), r = L.r[s];
            const float t1 = kMgOmega * di * r;
            const float nb = mg_nb_sum(i, j, k, L.D, L.cell, [&](uint32_t u) { return kMgOmega * mg_dinv(L.cell[u]) * L.r[u]; });
            const float at = (float)(c & 7u) * t1 - nb;
            out = t1 + kMgOmega * di * (r - at);
        }
        L.t[s] = out;
    }
}

// residual r - A t on level F, restricted to C: C.r[parent] = 1/2 sum over
// the children (fluid parents only).  C.r is cleared beforehand (parents of
// tiles outside F's list keep 0).
__global__ void __launch_bounds__(512) mg_restrict_kernel(MgLevel F, MgLevel C, const int* halt) {
    if (mg_halted(halt)) return;
    __shared__ float S[512];
    const uint32_t n = *F.d_ntiles;
    for (uint32_t tt = blockIdx.x; tt < n; tt += gridDim.x) {
        const uint32_t key = F.tiles[tt];
        const uint32_t s = (key << 9) | threadIdx.x;
        const uint8_t c = F.cell[s];
        int i, j, k;
        mg_cell_of(key, threadIdx.x, F.D, i, j, k);
        float res = 0.0f;
        if (c & kCellFluid) {
            const float nb = mg_nb_sum(i, j, k, F.D, F.cell, [&](uint32_t u) { return F.t[u]; });
            res = F.r[s] - ((float)(c & 7u) * F.t[s] - nb);
        }
        S[threadIdx.x] = res;
        __syncthreads();
        if ((threadIdx.x & 0x49u) == 0) {  // the (even, even, even) child of each 2^3 block
            const int b = threadIdx.x;
            const float sum = ((S[b] + S[b + 1]) + (S[b + 8] + S[b + 9])) + ((S[b + 64] + S[b + 65]) + (S[b + 72] + S[b + 73]));
            const uint32_t p = mg_slot(i >> 1, j >> 1, k >> 1, C.D);
            C.r[p] = (C.cell[p] & kCellFluid) ? 0.5f * sum : 0.0f;
        }
        __syncthreads();
    }
}

// prolongation and the first post-smoothing sweep: u = t + P e (e = C.z, the
// parent's value on fluid cells), t2 = u + w D^-1 (r - A u)
__global__ void __launch_bounds__(512) mg_post_kernel(MgLevel F, MgLevel C, const int* halt) {
    if (mg_halted(halt)) return;
    const uint32_t n = *F.d_ntiles;
    for (uint32_t tt = blockIdx.x; tt < n; tt += gridDim.x) {
        const uint32_t key = F.tiles[tt];
        const uint32_t s = (key << 9) | threadIdx.x;
        const uint8_t c = F.cell[s];
        float out = 0.0f;
        if (c & kCellFluid) {
            int i, j, k;
            mg_cell_of(key, threadIdx.x, F.D, i, j, k);
            auto u_at = [&](uint32_t u, int a, int b, int cc) { return F.t[u] + C.z[mg_slot(a >> 1, b >> 1, cc >> 1, C.D)]; };
            const float us = u_at(s, i, j, k);
            const int oi[6] = {-1, 1, 0, 0, 0, 0}, oj[6] = {0, 0, -1, 1, 0, 0}, ok[6] = {0, 0, 0, 0, -1, 1};
            float nb = 0.0f;
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                const int a = i + oi[q], b = j + oj[q], cc = k + ok[q];
                if (!mg_in(a, b, cc, F.D)) continue;
                const uint32_t u = mg_slot(a, b, cc, F.D);
                if (F.cell[u] & kCellFluid) nb += u_at(u, a, b, cc);
            }
            out = us + kMgOmega * mg_dinv(c) * (F.r[s] - ((float)(c & 7u) * us - nb));
        }
        F.t2[s] = out;
    }
}

// one damped Jacobi sweep: out = in + w D^-1 (r - A in)
__global__ void __launch_bounds__(512) mg_smooth_kernel(MgLevel L, const float* __restrict__ in, float* __restrict__ out,
                                                        const int* halt) {
    if (mg_halted(halt)) return;
    const uint32_t n = *L.d_ntiles;
    for (uint32_t tt = blockIdx.x; tt < n; tt += gridDim.x) {
        const uint32_t key = L.tiles[tt];
        const uint32_t s = (key << 9) | threadIdx.x;
        const uint8_t c = L.cell[s];
        float v = 0.0f;
        if (c & kCellFluid) {
            int i, j, k;
            mg_cell_of(key, threadIdx.x, L.D, i, j, k);
            const float nb = mg_nb_sum(i, j, k, L.D, L.cell, [&](uint32_t u) { return in[u]; });
            const float x = in[s];
            v = x + kMgOmega * mg_dinv(c) * (L.r[s] - ((float)(c & 7u) * x - nb));
        }
        out[s] = v;
    }
}

// coarsest start: z = zn + D^-1 r with the network output zn, else w D^-1 r
__global__ void __launch_bounds__(512) mg_coarse_start_kernel(MgLevel L, const float* __restrict__ zn, float* __restrict__ out,
                                                              const int* halt) {
    if (mg_halted(halt)) return;
    const uint32_t n = *L.d_ntiles;
    for (uint32_t tt = blockIdx.x; tt < n; tt += gridDim.x) {
        const uint32_t s = (L.tiles[tt] << 9) | threadIdx.x;
        const uint8_t c = L.cell[s];
        float v = 0.0f;
        if (c & kCellFluid) v = zn ? zn[s] + mg_dinv(c) * L.r[s] : kMgOmega * mg_dinv(c) * L.r[s];
        out[s] = v;
    }
}

// 1 / rms(r) over the fluid cells of a level (one CTA)
__global__ void __launch_bounds__(1024) mg_scale_kernel(MgLevel L, float* inv_s, const int* halt) {
    if (mg_halted(halt)) return;
    __shared__ double sh[32];
    const uint32_t n = *L.d_ntiles;
    double rr = 0.0, nf = 0.0;
    for (uint32_t v = threadIdx.x; v < n * 512u; v += 1024u) {
        const uint32_t s = (L.tiles[v >> 9] << 9) | (v & 511u);
        if (L.cell[s] & kCellFluid) {
            const double r = L.r[s];
            rr += r * r;
            nf += 1.0;
        }
    }
    rr = block_sum_f64<1024>(rr, sh);
    __syncthreads();
    nf = block_sum_f64<1024>(nf, sh);
    if (threadIdx.x == 0) *inv_s = rr > 0.0 ? (float)(1.0 / sqrt(rr / fmax(nf, 1.0))) : 1.0f;
}

// Jacobi-PCG on one level in one CTA (the coarsest level: at most 4096
// slots): x = A^-1 b to |r| <= tol |b| or max_iter iterations, FP32 vectors
// and FP64 dots.  r, p, q are scratch vectors of the level's size.  Used for
// the training targets of the coarsest solve.
__global__ void __launch_bounds__(1024) mg_cg_kernel(MgLevel L, const float* __restrict__ b, float* __restrict__ x,
                                                     float* __restrict__ r, float* __restrict__ p, float* __restrict__ q,
                                                     double tol, int max_iter, int* iters) {
    __shared__ double sh[32];
    __shared__ double bc;
    const uint32_t n = *L.d_ntiles * 512u;
    auto slot = [&](uint32_t v) { return (L.tiles[v >> 9] << 9) | (v & 511u); };
    auto bsum = [&](double v) {
        v = block_sum_f64<1024>(v, sh);
        if (threadIdx.x == 0) bc = v;
        __syncthreads();
        return bc;
    };
    double bb = 0.0, rz = 0.0;
    for (uint32_t v = threadIdx.x; v < n; v += 1024u) {
        const uint32_t s = slot(v);
        const uint8_t c = L.cell[s];
        const float bv = (c & kCellFluid) ? b[s] : 0.0f;
        x[s] = 0.0f;
        r[s] = bv;
        const float z = mg_dinv(c) * bv;
        p[s] = z;
        bb += (double)bv * bv;
        rz += (double)bv * z;
    }
    bb = bsum(bb);
    rz = bsum(rz);
    int it = 0;
    if (bb > 0.0) {
        for (it = 1; it <= max_iter; ++it) {
            double pq = 0.0;
            for (uint32_t v = threadIdx.x; v < n; v += 1024u) {
                const uint32_t s = slot(v);
                const uint8_t c = L.cell[s];
                float qv = 0.0f;
                if (c & kCellFluid) {
                    int i, j, k;
                    mg_cell_of(s >> 9, (int)(s & 511u), L.D, i, j, k);
                    const float nb = mg_nb_sum(i, j, k, L.D, L.cell, [&](uint32_t u) { return p[u]; });
                    qv = (float)(c & 7u) * p[s] - nb;
                }
                q[s] = qv;
                pq += (double)p[s] * qv;
            }
            pq = bsum(pq);
            if (!(pq > 0.0)) break;
            const float alpha = (float)(rz / pq);
            double rr = 0.0, rzn = 0.0;
            for (uint32_t v = threadIdx.x; v < n; v += 1024u) {
                const uint32_t s = slot(v);
                x[s] += alpha * p[s];
                const float rv = r[s] - alpha * q[s];
                r[s] = rv;
                rr += (double)rv * rv;
                rzn += (double)rv * (mg_dinv(L.cell[s]) * rv);
            }
            rr = bsum(rr);
            rzn = bsum(rzn);
            if (rr <= tol * tol * bb) break;
            const float beta = (float)(rzn / rz);
            rz = rzn;
            for (uint32_t v = threadIdx.x; v < n; v += 1024u) {
                const uint32_t s = slot(v);
                p[s] = mg_dinv(L.cell[s]) * r[s] + beta * p[s];
            }
            __syncthreads();
        }
    }
    if (threadIdx.x == 0 && iters) *iters = it;
}

// ------------------------------------------------------------ host side
int mg_plan(int nx, int ny, int nz, float h, MgLevel* L, int max_levels) {
    int ex = nx, ey = ny, ez = nz, levels = 0;
    float hl = h;
    while (levels < max_levels) {
        MgLevel& l = L[levels];
        l = MgLevel{};
        l.ex = ex; l.ey = ey; l.ez = ez;
        l.D.nx = (ex + 7) & ~7; l.D.ny = (ey + 7) & ~7; l.D.nz = (ez + 7) & ~7;
        l.D.tx = l.D.nx / 8; l.D.ty = l.D.ny / 8; l.D.tz = l.D.nz / 8;
        l.D.ox = l.D.oy = l.D.oz = 0.0f;
        l.D.h = hl;
        l.ntiles = (uint32_t)(l.D.tx * l.D.ty * l.D.tz);
        ++levels;
        if (ex <= kMgCoarsest && ey <= kMgCoarsest && ez <= kMgCoarsest) break;
        ex = (ex + 1) / 2; ey = (ey + 1) / 2; ez = (ez + 1) / 2;
        hl *= 2.0f;
    }
    return levels;
}

static int mg_grid(const MgLevel& L, int grid0, int level) {
    if (level == 0) return grid0;
    return (int)(L.ntiles < 1184u ? L.ntiles : 1184u);
}

int mg_build(const MgHierarchy& H, const int* halt, cudaStream_t s) {
    for (int l = 1; l < H.levels; ++l) {
        const int g = (int)((H.L[l].ntiles + 0u) < 1184u ? H.L[l].ntiles : 1184u);
        mg_coarsen_kernel<<<g, 512, 0, s>>>(H.L[l - 1], H.L[l], halt);
        mg_codes_kernel<<<g, 512, 0, s>>>(H.L[l], halt);
    }
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int mg_down(const MgHierarchy& H, const int* halt, int grid0, cudaStream_t s) {
    for (int l = 0; l + 1 < H.levels; ++l) {
        const MgLevel &F = H.L[l], &C = H.L[l + 1];
        mg_pre_kernel<<<mg_grid(F, grid0, l), 512, 0, s>>>(F, halt);
        FLIP_CUDA_TRY(cudaMemsetAsync(C.r, 0, (size_t)C.ntiles * 512u * sizeof(float), s));
        mg_restrict_kernel<<<mg_grid(F, grid0, l), 512, 0, s>>>(F, C, halt);
    }
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int mg_coarsest(const MgHierarchy& H, const float* zn, const int* halt, cudaStream_t s) {
    const MgLevel& L = H.L[H.levels - 1];
    const int g = mg_grid(L, 1184, H.levels - 1);
    mg_coarse_start_kernel<<<g, 512, 0, s>>>(L, zn, L.z, halt);
    mg_smooth_kernel<<<g, 512, 0, s>>>(L, L.z, L.t, halt);
    mg_smooth_kernel<<<g, 512, 0, s>>>(L, L.t, L.z, halt);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int mg_up(const MgHierarchy& H, const int* halt, int grid0, cudaStream_t s) {
    for (int l = H.levels - 2; l >= 0; --l) {
        const MgLevel &F = H.L[l], &C = H.L[l + 1];
        const int g = mg_grid(F, grid0, l);
        mg_post_kernel<<<g, 512, 0, s>>>(F, C, halt);
        mg_smooth_kernel<<<g, 512, 0, s>>>(F, F.t2, F.z, halt);
    }
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int mg_cg(const MgLevel& L, const float* b, float* x, float* r, float* p, float* q, double tol, int max_iter, int* iters,
          cudaStream_t s) {
    mg_cg_kernel<<<1, 1024, 0, s>>>(L, b, x, r, p, q, tol, max_iter, iters);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

int mg_input_scale(const MgHierarchy& H, const int* halt, cudaStream_t s) {
    mg_scale_kernel<<<1, 1024, 0, s>>>(H.L[H.levels - 1], H.inv_s, halt);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

}  // namespace flip
