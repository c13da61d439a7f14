// pcg_tma.cu -- the Jacobi-PCG iteration with tiles staged by TMA (sm_100a).
//
// The iteration is two kernels, as in native.cu: the direction update fused
// with the matvec (p' = D^-1 r + beta p, q = A p', p'.q), then the update
// (xg += alpha p', r -= alpha q, r.r, r.D^-1 r).  These forms keep several
// tiles in flight per CTA without spending registers on them: one thread
// issues cp.async.bulk.tensor loads of a tile's vectors into a ring of
// shared-memory stages a few tiles ahead of the 128 threads that compute,
// and each stage completes on its own mbarrier (bounded waits).
//
// The residual is kept Jacobi-scaled, w = D^-1 r (d = the number of
// non-solid neighbours of a fluid cell).  Then p' = w + beta p needs no cell
// code, and w, p are zero on every non-fluid cell of the dilated tile list
// (pcg_init_kernel<true> zeroes them), so the halo of a tile -- the faces of
// its six neighbours -- is read without the neighbours' cell codes.  The
// update keeps w: w -= alpha D^-1 q, r.r = sum (d w)^2, r.z = sum d w^2.
//
// Tile-blocked vectors are viewed as 4-D tensors (8 x 8 x 8 x tiles).  Per
// tile a stage receives the tile's w and p (2 KiB each) and cell codes, and
// of each existing neighbour the face it needs: x faces as 4 x 8 x 8 boxes
// (a one-float x extent is below the 16-byte minimum; x = 4..7 of the -x
// neighbour and 0..3 of the +x neighbour, whose innermost coordinates 4 and
// 0 are 16-byte aligned), y faces as 8 x 1 x 8 and z faces as 8 x 8 x 1
// boxes.  A thread owns four consecutive x cells of one (y, z) row and reads
// every neighbour value it needs from the stage, so no barrier separates the
// direction update from the stencil.  Only plain (non-multicast) loads of
// this GPU's own buffers are issued.
#include "common.cuh"
#include "native.cuh"
#include "tma.cuh"

namespace flip {

namespace {
constexpr int kPtThreads = 128;
constexpr int kPtStages = 4;
constexpr uint32_t kPtSpinLimit = 1u << 24;

struct MatvecStage {  // 10,752 bytes; every array starts on a 256-byte boundary
    float w[512], p[512];          // the tile
    float wx[2][256], px[2][256];  // -x neighbour x = 4..7, +x neighbour x = 0..3: [z][y][4]
    float wy[2][64], py[2][64];    // -y neighbour row y = 7, +y row y = 0: [z][x]
    float wz[2][64], pz[2][64];    // -z neighbour plane z = 7, +z plane z = 0: [y][x]
    uint8_t cell[512];
};
struct UpdateStage {  // 8,704 bytes
    float p[512], q[512], w[512], g[512];
    uint8_t cell[512];
};
constexpr uint32_t kMvSmem = kPtStages * sizeof(MatvecStage) + 64;
constexpr uint32_t kUpSmem = kPtStages * sizeof(UpdateStage) + 64;

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, int t, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(t), "r"(smem_addr(bar))
        : "memory");
}

struct Nb {  // which of the six face neighbours exist
    bool xm, xp, ym, yp, zm, zp;
};
__device__ __forceinline__ Nb neighbours(uint32_t tc, const NatDims& D) {
    const int tx = (int)(tc & 1023u), ty = (int)((tc >> 10) & 1023u), tz = (int)(tc >> 20);
    return Nb{tx > 0, tx < D.tx - 1, ty > 0, ty < D.ty - 1, tz > 0, tz < D.tz - 1};
}

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ float4 dir4(const float4& w, const float4& p, float beta) {
    return make_float4(fmaf(beta, p.x, w.x), fmaf(beta, p.y, w.y), fmaf(beta, p.z, w.z), fmaf(beta, p.w, w.w));
}
}  // namespace

// ------------------------------------------------- direction + matvec
__global__ void __launch_bounds__(kPtThreads) pcgw_matvec_kernel(const __grid_constant__ PcgMaps M,
                                                                 const uint32_t* __restrict__ tiles,
                                                                 const uint32_t* __restrict__ tcoord,
                                                                 const uint32_t* __restrict__ d_ntiles, NatDims D,
                                                                 float* p0, float* p1, float* __restrict__ q,
                                                                 double* __restrict__ x, float* __restrict__ xg,
                                                                 PcgState* st, double* partials, uint32_t* err) {
    if (st->done || st->pending) return;
    extern __shared__ __align__(128) unsigned char mv_smem[];
    MatvecStage* S = reinterpret_cast<MatvecStage*>(mv_smem);
    uint64_t* bar = reinterpret_cast<uint64_t*>(mv_smem + kPtStages * sizeof(MatvecStage));
    __shared__ double sh[32];
    const int tid = threadIdx.x;
    const uint32_t ntiles = *d_ntiles;
    const bool pc = st->pcur != 0;
    float* pn = pc ? p0 : p1;  // this iteration's direction goes to the other buffer
    const CUtensorMap* mp[4] = {pc ? &M.p1c : &M.p0c, pc ? &M.p1x : &M.p0x, pc ? &M.p1y : &M.p0y, pc ? &M.p1z : &M.p0z};
    const float beta = (float)st->beta;
    const bool flush = st->flush != 0;
    if (tid == 0)
        for (int s = 0; s < kPtStages; ++s) mbar_init(&bar[s], 1);
    __syncthreads();

    // producer (thread 0): the loads of this CTA's k-th tile into stage k % kPtStages
    auto issue = [&](uint32_t k) {
        const uint32_t t = blockIdx.x + k * gridDim.x;
        if (t >= ntiles) return;
        MatvecStage& T = S[k % kPtStages];
        uint64_t* b = &bar[k % kPtStages];
        const int key = (int)tiles[t];
        const Nb nb = neighbours(tcoord[t], D);
        uint32_t bytes = 2 * 2048 + 512;
        bytes += (nb.xm + nb.xp) * 2u * 1024u + (nb.ym + nb.yp + nb.zm + nb.zp) * 2u * 256u;
        fence_proxy_async_smem();
        mbar_expect_tx(b, bytes);
        tma_load_4d(T.w, &M.wc, 0, 0, 0, key, b);
        tma_load_4d(T.p, mp[0], 0, 0, 0, key, b);
        tma_load_4d(T.cell, &M.cellc, 0, 0, 0, key, b);
        const int dy = D.tx, dz = D.tx * D.ty;
        if (nb.xm) { tma_load_4d(T.wx[0], &M.wx, 4, 0, 0, key - 1, b); tma_load_4d(T.px[0], mp[1], 4, 0, 0, key - 1, b); }
        if (nb.xp) { tma_load_4d(T.wx[1], &M.wx, 0, 0, 0, key + 1, b); tma_load_4d(T.px[1], mp[1], 0, 0, 0, key + 1, b); }
        if (nb.ym) { tma_load_4d(T.wy[0], &M.wy, 0, 7, 0, key - dy, b); tma_load_4d(T.py[0], mp[2], 0, 7, 0, key - dy, b); }
        if (nb.yp) { tma_load_4d(T.wy[1], &M.wy, 0, 0, 0, key + dy, b); tma_load_4d(T.py[1], mp[2], 0, 0, 0, key + dy, b); }
        if (nb.zm) { tma_load_4d(T.wz[0], &M.wz, 0, 0, 7, key - dz, b); tma_load_4d(T.pz[0], mp[3], 0, 0, 7, key - dz, b); }
        if (nb.zp) { tma_load_4d(T.wz[1], &M.wz, 0, 0, 0, key + dz, b); tma_load_4d(T.pz[1], mp[3], 0, 0, 0, key + dz, b); }
    };
    if (tid == 0)
        for (uint32_t k = 0; k < (uint32_t)kPtStages; ++k) issue(k);

    // consumer: a thread owns cells x0..x0+3 of row (y, z)
    const int row = tid >> 1, x0 = 4 * (tid & 1), y = row & 7, z = row >> 3;
    const int base = x0 + 8 * y + 64 * z;
    const int xh = 4 * (y + 8 * z);  // the row in an x-face box
    double pq = 0.0;
    for (uint32_t k = 0;; ++k) {
        const uint32_t t = blockIdx.x + k * gridDim.x;
        if (t >= ntiles) break;
        const int s = (int)(k % kPtStages);
        // every thread waits on the stage; the CTA decides together
        if (!__syncthreads_and(mbar_wait_bounded(&bar[s], (k / kPtStages) & 1u, kPtSpinLimit))) {
            // the copies never completed: report, let any copy in flight land
            // (bounded), and leave; the solve ends with the error flag set
            if (tid == 0) atomicOr(err, DEVERR_TMA_TIMEOUT);
            mbar_wait_bounded(&bar[s], (k / kPtStages) & 1u, kPtSpinLimit);
            return;
        }
        const MatvecStage& T = S[s];
        const Nb nb = neighbours(tcoord[t], D);
        const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const float4 pc4 = dir4(ld4(T.w + base), ld4(T.p + base), beta);
        float4 ym, yp, zm, zp;
        if (y > 0) ym = dir4(ld4(T.w + base - 8), ld4(T.p + base - 8), beta);
        else ym = nb.ym ? dir4(ld4(T.wy[0] + 8 * z + x0), ld4(T.py[0] + 8 * z + x0), beta) : zero4;
        if (y < 7) yp = dir4(ld4(T.w + base + 8), ld4(T.p + base + 8), beta);
        else yp = nb.yp ? dir4(ld4(T.wy[1] + 8 * z + x0), ld4(T.py[1] + 8 * z + x0), beta) : zero4;
        if (z > 0) zm = dir4(ld4(T.w + base - 64), ld4(T.p + base - 64), beta);
        else zm = nb.zm ? dir4(ld4(T.wz[0] + 8 * y + x0), ld4(T.pz[0] + 8 * y + x0), beta) : zero4;
        if (z < 7) zp = dir4(ld4(T.w + base + 64), ld4(T.p + base + 64), beta);
        else zp = nb.zp ? dir4(ld4(T.wz[1] + 8 * y + x0), ld4(T.pz[1] + 8 * y + x0), beta) : zero4;
        float xl, xr;
        if (x0 == 4) xl = fmaf(beta, T.p[base - 1], T.w[base - 1]);
        else xl = nb.xm ? fmaf(beta, T.px[0][xh + 3], T.wx[0][xh + 3]) : 0.0f;
        if (x0 == 0) xr = fmaf(beta, T.p[base + 4], T.w[base + 4]);
        else xr = nb.xp ? fmaf(beta, T.px[1][xh], T.wx[1][xh]) : 0.0f;
        const uint32_t c4 = *reinterpret_cast<const uint32_t*>(T.cell + base);
        const float pv[4] = {pc4.x, pc4.y, pc4.z, pc4.w};
        const float yl[4] = {ym.x, ym.y, ym.z, ym.w}, yr[4] = {yp.x, yp.y, yp.z, yp.w};
        const float zl[4] = {zm.x, zm.y, zm.z, zm.w}, zr[4] = {zp.x, zp.y, zp.z, zp.w};
        float qv[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const uint8_t c = (uint8_t)(c4 >> (8 * m));
            const float l = m == 0 ? xl : pv[m - 1], r = m == 3 ? xr : pv[m + 1];
            float qc = 0.0f;
            if (c & kCellFluid) qc = fmaf((float)(c & 7u), pv[m], -(((l + r) + (yl[m] + yr[m])) + (zl[m] + zr[m])));
            qv[m] = qc;
            pq += (double)pv[m] * (double)qc;
        }
        const uint32_t sg = ((uint32_t)tiles[t] << 9) | (uint32_t)base;
        *reinterpret_cast<float4*>(pn + sg) = pc4;
        *reinterpret_cast<float4*>(q + sg) = make_float4(qv[0], qv[1], qv[2], qv[3]);
        if (flush && c4) {
#pragma unroll
            for (int m = 0; m < 4; ++m)
                if ((c4 >> (8 * m)) & kCellFluid) {
                    x[sg + m] += (double)xg[sg + m];
                    xg[sg + m] = 0.0f;
                }
        }
        __syncthreads();  // the stage is free: every thread has read it
        if (tid == 0) issue(k + kPtStages);
    }
    double vals[1] = {pq}, out[1];
    if (last_block_reduce_n<1, kPtThreads>(vals, partials, &st->ticket, sh, out) && tid == 0) {
        st->pq = out[0];
        st->flush = 0;
        if (out[0] > 0.0) st->alpha = st->rz / out[0];
        else { st->alpha = 0.0; st->done = 3; }  // breakdown
    }
}

// ------------------------------------------------------------- update
__global__ void __launch_bounds__(kPtThreads) pcgw_update_kernel(const __grid_constant__ PcgMaps M,
                                                                 const uint32_t* __restrict__ tiles,
                                                                 const uint32_t* __restrict__ d_ntiles, float* w,
                                                                 float* xg, PcgState* st, double* partials,
                                                                 uint32_t* err) {
    if (st->done || st->pending) return;
    extern __shared__ __align__(128) unsigned char up_smem[];
    UpdateStage* S = reinterpret_cast<UpdateStage*>(up_smem);
    uint64_t* bar = reinterpret_cast<uint64_t*>(up_smem + kPtStages * sizeof(UpdateStage));
    __shared__ double sh[32];
    const int tid = threadIdx.x;
    const uint32_t ntiles = *d_ntiles;
    const CUtensorMap* mp = st->pcur ? &M.p0c : &M.p1c;  // the direction the matvec just wrote
    const float a = (float)st->alpha;
    if (tid == 0)
        for (int s = 0; s < kPtStages; ++s) mbar_init(&bar[s], 1);
    __syncthreads();
    auto issue = [&](uint32_t k) {
        const uint32_t t = blockIdx.x + k * gridDim.x;
        if (t >= ntiles) return;
        UpdateStage& T = S[k % kPtStages];
        uint64_t* b = &bar[k % kPtStages];
        const int key = (int)tiles[t];
        fence_proxy_async_smem();
        mbar_expect_tx(b, 4 * 2048 + 512);
        tma_load_4d(T.p, mp, 0, 0, 0, key, b);
        tma_load_4d(T.q, &M.qc, 0, 0, 0, key, b);
        tma_load_4d(T.w, &M.wc, 0, 0, 0, key, b);
        tma_load_4d(T.g, &M.xgc, 0, 0, 0, key, b);
        tma_load_4d(T.cell, &M.cellc, 0, 0, 0, key, b);
    };
    if (tid == 0)
        for (uint32_t k = 0; k < (uint32_t)kPtStages; ++k) issue(k);
    const int base = 4 * tid;
    double rr = 0.0, rz = 0.0;
    for (uint32_t k = 0;; ++k) {
        const uint32_t t = blockIdx.x + k * gridDim.x;
        if (t >= ntiles) break;
        const int s = (int)(k % kPtStages);
        if (!__syncthreads_and(mbar_wait_bounded(&bar[s], (k / kPtStages) & 1u, kPtSpinLimit))) {
            if (tid == 0) atomicOr(err, DEVERR_TMA_TIMEOUT);
            mbar_wait_bounded(&bar[s], (k / kPtStages) & 1u, kPtSpinLimit);
            return;
        }
        const UpdateStage& T = S[s];
        const uint32_t c4 = *reinterpret_cast<const uint32_t*>(T.cell + base);
        if (c4) {
            const float4 w4 = ld4(T.w + base), g4 = ld4(T.g + base), p4 = ld4(T.p + base), q4 = ld4(T.q + base);
            float wv[4] = {w4.x, w4.y, w4.z, w4.w}, gv[4] = {g4.x, g4.y, g4.z, g4.w};
            const float pv[4] = {p4.x, p4.y, p4.z, p4.w}, qv[4] = {q4.x, q4.y, q4.z, q4.w};
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const uint8_t c = (uint8_t)(c4 >> (8 * m));
                if (!(c & kCellFluid)) continue;
                const float d = (float)(c & 7u);
                gv[m] = fmaf(a, pv[m], gv[m]);
                const float wn = fmaf(-a, __fdiv_rn(qv[m], d), wv[m]);
                wv[m] = wn;
                const float rs = d * wn;
                rr += (double)rs * (double)rs;
                rz += (double)rs * (double)wn;
            }
            const uint32_t sg = ((uint32_t)tiles[t] << 9) | (uint32_t)base;
            *reinterpret_cast<float4*>(w + sg) = make_float4(wv[0], wv[1], wv[2], wv[3]);
            *reinterpret_cast<float4*>(xg + sg) = make_float4(gv[0], gv[1], gv[2], gv[3]);
        }
        __syncthreads();
        if (tid == 0) issue(k + kPtStages);
    }
    double vals[2] = {rr, rz}, out[2];
    if (last_block_reduce_n<2, kPtThreads>(vals, partials, &st->ticket, sh, out) && tid == 0) {
        st->iter += 1;
        st->pcur ^= 1;
        st->rr = out[0];
        st->rz_prev = st->rz;
        st->rz = out[1];
        st->beta = st->rz / st->rz_prev;
        st->inv_s = out[0] > 0.0 ? (float)(1.0 / sqrt(out[0] / fmax(st->nfluid, 1.0))) : 1.0f;
        if (out[0] <= st->tol2 * st->bb) st->pending = 1;  // confirm with the true residual
        else if (st->iter >= st->max_iter) st->done = 2;
        st->halt = st->done || st->pending;
    }
}

int nat_launch_pcgw_iteration(const PcgMaps& M, const uint32_t* tiles, const uint32_t* d_ntiles, const NatDims& D,
                              PcgBuffers& B, uint32_t* err, int grid, cudaStream_t s) {
    static bool attr_done = false;
    if (!attr_done) {
        FLIP_CUDA_TRY(cudaFuncSetAttribute(pcgw_matvec_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kMvSmem));
        FLIP_CUDA_TRY(cudaFuncSetAttribute(pcgw_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kUpSmem));
        attr_done = true;
    }
    if (grid > kPcgBlocks) grid = kPcgBlocks;  // the partial sums hold kPcgBlocks values per quantity
    pcgw_matvec_kernel<<<grid, kPtThreads, kMvSmem, s>>>(M, tiles, B.tcoord, d_ntiles, D, B.p0, B.p1, B.q, B.x, B.xg,
                                                         B.st, B.partials, err);
    pcgw_update_kernel<<<grid, kPtThreads, kUpSmem, s>>>(M, tiles, d_ntiles, B.r, B.xg, B.st, B.partials, err);
    FLIP_CUDA_TRY(cudaGetLastError());
    return FLIP_OK;
}

// ------------------------------------------------------- tensor maps
int nat_make_pcg_maps(PcgMaps& M, const PcgBuffers& B, uint64_t ntiles_total) {
    const uint64_t nt = ntiles_total;
    auto f32 = [&](CUtensorMap* m, const float* base, uint32_t bx, uint32_t by, uint32_t bz) {
        const uint64_t dims[4] = {8, 8, 8, nt};
        const uint64_t strides[3] = {32, 256, 2048};
        const uint32_t box[4] = {bx, by, bz, 1};
        return encode_tensor_map(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, dims, strides, box);
    };
    struct V {
        const float* a;
        CUtensorMap *c, *x, *y, *z;
    };
    const V vs[3] = {{B.r, &M.wc, &M.wx, &M.wy, &M.wz}, {B.p0, &M.p0c, &M.p0x, &M.p0y, &M.p0z},
                     {B.p1, &M.p1c, &M.p1x, &M.p1y, &M.p1z}};
    for (const V& v : vs) {
        if (int rc = f32(v.c, v.a, 8, 8, 8)) return rc;
        if (int rc = f32(v.x, v.a, 4, 8, 8)) return rc;
        if (int rc = f32(v.y, v.a, 8, 1, 8)) return rc;
        if (int rc = f32(v.z, v.a, 8, 8, 1)) return rc;
    }
    if (int rc = f32(&M.qc, B.q, 8, 8, 8)) return rc;
    if (int rc = f32(&M.xgc, B.xg, 8, 8, 8)) return rc;
    // cell codes: 16-byte rows of two x-rows each, 512 bytes a tile
    const uint64_t cdims[4] = {16, 4, 8, nt};
    const uint64_t cstrides[3] = {16, 64, 512};
    const uint32_t cbox[4] = {16, 4, 8, 1};
    return encode_tensor_map(&M.cellc, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, B.cell, cdims, cstrides, cbox);
}

}  // namespace flip
