/*
 * flip_oracle.c -- CPU restatement of the flip2 fluid step.  TEST
 * INFRASTRUCTURE ONLY: the parity checker for the CUDA path (tests/, the
 * smoke check) and the timed CPU baseline (bench.py).  The product library
 * never links or calls it.
 *
 * Build: gcc -O2 -fopenmp -ffp-contract=off -fPIC -shared (oracle/Makefile).
 * -ffp-contract=off keeps every product rounded on its own; where the CUDA
 * compiler contracts a multiply-add in the reference source (nvcc's default
 * --fmad=true), this file writes the fma() explicitly so the rounding matches.
 *
 * Citations are path:line inside the reference project (Aidan-F-Ryan/flip2).
 * Integer conversions follow the GPU's saturating cvt.rzi semantics
 * (negative -> 0, NaN -> 0), which is what the reference's `uint x = floor(..)`
 * does on the device.
 */
#include "flip_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

#define NV1D 8u          /* numVoxels1D = 2*floor(radius) + (2<<refinementLevel), particles.cu:37 */
#define NVPN 512u        /* numVoxelsPerNode */
#define APRON 2u         /* floor(radius), radius = 2 (particles.cu:17) */

/* ------------------------------------------------------------- helpers */
static inline uint32_t sat_u32_d(double v) {
    if (!(v > 0.0)) return 0u;               /* NaN and negatives -> 0 */
    if (v >= 4294967295.0) return 0xFFFFFFFFu;
    return (uint32_t)v;
}
static inline uint32_t sat_u32_f(float v) {
    if (!(v > 0.0f)) return 0u;
    if (v >= 4294967295.0f) return 0xFFFFFFFFu;
    return (uint32_t)v;
}
/* distance() (particles.cu:84-86) */
static inline double ref_dist(double dx, double dy, double dz) {
    return sqrt(fma(dx, dx, fma(dy, dy, dz * dz)));
}
/* calcSubCellWidth (voxelSolveFunctions.hu:10-12): float division by 4 */
static inline double ref_scw(orc_grid g) { return (double)(g.cellSize / 4.0f); }
/* (p - neg - gid*cell + apron*scw) (particles.cu:140-142): the product
 * gid*cellSize is a float multiply (uint * float). */
static inline double ref_local(double p, float neg, uint32_t gid, float cell, double scw) {
    double t = p - (double)neg;
    float prod = (float)gid * cell;
    t = t - (double)prod;
    return t + 2.0 * scw;
}
static inline void ref_decompose(uint32_t key, orc_grid g, uint32_t* gx, uint32_t* gy, uint32_t* gz) {
    uint32_t xy = g.sizeX * g.sizeY;
    uint32_t m = key % xy;
    *gz = key / xy;
    *gy = m / g.sizeX;
    *gx = m % g.sizeX;
}

/* ------------------------------------------------------------- binning */
void orc_ref_keys(int64_t n, double* px, double* py, double* pz, orc_grid g, uint32_t* keys) {
    /* upper face: grid.negX + grid.sizeX*grid.cellSize, a float multiply-add */
    float ux = fmaf((float)g.sizeX, g.cellSize, g.negX);
    float uy = fmaf((float)g.sizeY, g.cellSize, g.negY);
    float uz = fmaf((float)g.sizeZ, g.cellSize, g.negZ);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double x = px[i], y = py[i], z = pz[i];
        if (x < (double)g.negX) x = g.negX; else if (x > (double)ux) x = ux;
        if (y < (double)g.negY) y = g.negY; else if (y > (double)uy) y = uy;
        if (z < (double)g.negZ) z = g.negZ; else if (z > (double)uz) z = uz;
        px[i] = x; py[i] = y; pz[i] = z;
        /* floorf takes the double quotient narrowed to float (Q1) */
        uint32_t kx = sat_u32_f(floorf((float)((x - (double)g.negX) / (double)g.cellSize)));
        uint32_t ky = sat_u32_f(floorf((float)((y - (double)g.negY) / (double)g.cellSize)));
        uint32_t kz = sat_u32_f(floorf((float)((z - (double)g.negZ) / (double)g.cellSize)));
        keys[i] = kx + ky * g.sizeX + kz * g.sizeX * g.sizeY;
    }
}

void orc_sort_pairs_payload(int64_t n, const uint32_t* keys_in, const uint32_t* vals_in,
                            uint32_t* keys_out, uint32_t* vals_out) {
    /* stable LSD counting sort, 8-bit digits; any stable sort gives the same
     * (keys, payload) as the reference's 32-pass 1-bit split sort. */
    uint32_t* ka = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
    uint32_t* va = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
    uint32_t* kb = keys_out;
    uint32_t* vb = vals_out;
    memcpy(ka, keys_in, sizeof(uint32_t) * (size_t)n);
    memcpy(va, vals_in, sizeof(uint32_t) * (size_t)n);
    for (int pass = 0; pass < 4; ++pass) {
        int sh = pass * 8;
        int64_t cnt[257];
        memset(cnt, 0, sizeof(cnt));
        for (int64_t i = 0; i < n; ++i) cnt[((ka[i] >> sh) & 0xFF) + 1]++;
        int trivial = 0;
        for (int d = 0; d < 256; ++d) if (cnt[d + 1] == n) trivial = 1;
        if (trivial) continue;
        for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
        for (int64_t i = 0; i < n; ++i) {
            uint32_t d = (ka[i] >> sh) & 0xFF;
            int64_t o = cnt[d]++;
            kb[o] = ka[i];
            vb[o] = va[i];
        }
        memcpy(ka, kb, sizeof(uint32_t) * (size_t)n);
        memcpy(va, vb, sizeof(uint32_t) * (size_t)n);
    }
    memcpy(keys_out, ka, sizeof(uint32_t) * (size_t)n);
    memcpy(vals_out, va, sizeof(uint32_t) * (size_t)n);
    free(ka);
    free(va);
}

void orc_sort_pairs(int64_t n, const uint32_t* keys_in, uint32_t* keys_out, uint32_t* perm_out) {
    uint32_t* idx = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
    for (int64_t i = 0; i < n; ++i) idx[i] = (uint32_t)i;
    orc_sort_pairs_payload(n, keys_in, idx, keys_out, perm_out);
    free(idx);
}

void orc_inclusive_scan(int64_t n, uint32_t* a) {
    uint32_t s = 0;
    for (int64_t i = 0; i < n; ++i) { s += a[i]; a[i] = s; }
}

uint32_t orc_exclusive_scan_small(uint32_t n, uint32_t* a) {
    uint32_t s = 0;
    for (uint32_t i = 0; i < n; ++i) { uint32_t v = a[i]; a[i] = s; s += v; }
    return s;
}

void orc_gather_f64(int64_t n, const uint32_t* perm, const double* in, double* out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) out[i] = in[perm[i]];
}

uint32_t orc_mark_unique_scan(int64_t n, const uint32_t* k, uint32_t* fs) {
    if (n <= 0) return 0;
    fs[0] = 1;
    for (int64_t i = 1; i < n; ++i) fs[i] = (k[i] != k[i - 1]) ? 1u : 0u;
    orc_inclusive_scan(n, fs);
    return fs[n - 1];
}

void orc_cell_starts(int64_t n, const uint32_t* fs, uint32_t* starts) {
    if (n <= 0) return;
    starts[0] = 0;
    for (int64_t i = 1; i < n; ++i)
        if (fs[i] != fs[i - 1]) starts[fs[i] - 1] = (uint32_t)i;
}

void orc_ydim_rows(uint32_t nodes, const uint32_t* starts, const uint32_t* keys, orc_grid g, uint32_t* table) {
    uint32_t rows = g.sizeY * g.sizeZ;
    for (uint32_t r = 0; r < rows; ++r) table[r] = nodes;
    for (uint32_t idx = 0; idx < nodes; ++idx) {
        uint32_t prev = idx ? keys[starts[idx - 1]] : nodes;   /* index 0 compares against the node count */
        uint32_t cur = keys[starts[idx]];
        uint32_t pr = prev / g.sizeX, cr = cur / g.sizeX;
        if (pr != cr && cr < rows) table[cr] = cur;            /* stores a cell id, not a node index (Q7) */
    }
}

/* Marks of one node's 8^3 tile (getNumberVoxelsUsedPerNode and
 * generateVoxelIDs share the predicate, particles.cu:111-178, 225-295). */
static void ref_node_marks(uint32_t b, uint32_t nodes, int64_t n, const uint32_t* starts, const uint32_t* keys,
                           const double* px, const double* py, const double* pz, orc_grid g,
                           uint32_t* mark, int8_t* solid) {
    memset(mark, 0, sizeof(uint32_t) * NVPN);
    if (solid) memset(solid, 0, NVPN);
    uint32_t gx, gy, gz;
    ref_decompose(keys[b], g, &gx, &gy, &gz);            /* tile origin from particle b's key (Q3) */
    const double fr = 2.0;                               /* floor(radius) */
    for (uint32_t i = 0; i < NVPN; ++i) {
        uint32_t vx = i % NV1D;
        uint32_t vy = (i % NV1D * NV1D) / NV1D;            /* precedence as written: equals vx (Q3) */
        uint32_t vz = i / (NV1D * NV1D);
        uint32_t gvx = gx * NV1D + vx, gvy = gy * NV1D + vy, gvz = gz * NV1D + vz;
        int s = 0;
        if ((double)gvx < fr || (double)gvy < fr || (double)gvz < fr) s = 1;
        else if ((double)gvx > (double)(g.sizeX * NV1D) + fr || (double)gvy > (double)(g.sizeY * NV1D) + fr ||
                 (double)gvz > (double)(g.sizeZ * NV1D) + fr) s = 1;
        if (s) { mark[i] = 1; if (solid) solid[i] = 1; }
    }
    uint32_t last = (b == nodes - 1) ? (uint32_t)n : starts[b + 1];
    double scw = ref_scw(g), hs = scw / 2.0, R = 2.0 * scw;
    for (uint32_t idx = starts[b]; idx < last; ++idx) {
        uint32_t qx, qy, qz;
        ref_decompose(keys[idx], g, &qx, &qy, &qz);
        double lx = ref_local(px[idx], g.negX, qx, g.cellSize, scw);
        double ly = ref_local(py[idx], g.negY, qy, g.cellSize, scw);
        double lz = ref_local(pz[idx], g.negZ, qz, g.cellSize, scw);
        uint32_t sx = sat_u32_d(floor(lx / scw)), sy = sat_u32_d(floor(ly / scw)), sz = sat_u32_d(floor(lz / scw));
        /* `int x = sx - apron; x < sx + apron` compares as unsigned */
        for (int x = (int)(sx - APRON); (uint32_t)x < sx + APRON; ++x)
            for (int y = (int)(sy - APRON); (uint32_t)y < sy + APRON; ++y)
                for (int z = (int)(sz - APRON); (uint32_t)z < sz + APRON; ++z) {
                    double dx = lx - x * scw, dy = ly - y * scw, dz = lz - z * scw;
                    double xc = ref_dist(dx, dy + hs, dz + hs);
                    double yc = ref_dist(dx + hs, dy, dz + hs);
                    double zc = ref_dist(dx + hs, dy + hs, dz);
                    if (xc < R || yc < R || zc < R)
                        if ((uint32_t)x < NV1D && (uint32_t)y < NV1D && (uint32_t)z < NV1D)
                            mark[x + y * NV1D + z * NV1D * NV1D] = 1;
                }
    }
}

void orc_ref_voxel_counts(uint32_t nodes, int64_t n, const uint32_t* starts, const uint32_t* keys,
                          const double* px, const double* py, const double* pz, orc_grid g, uint32_t* counts) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t b = 0; b < (int64_t)nodes; ++b) {
        uint32_t mark[NVPN];
        ref_node_marks((uint32_t)b, nodes, n, starts, keys, px, py, pz, g, mark, NULL);
        uint32_t c = 0;
        for (uint32_t i = 0; i < NVPN; ++i) c += mark[i];
        counts[b] = c;
    }
}

void orc_ref_voxel_ids(uint32_t nodes, int64_t n, const uint32_t* starts, const uint32_t* keys,
                       const double* px, const double* py, const double* pz, orc_grid g,
                       const uint32_t* node_voxels, uint32_t* voxel_ids, int8_t* solids) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t b = 0; b < (int64_t)nodes; ++b) {
        uint32_t mark[NVPN];
        int8_t sol[NVPN];
        ref_node_marks((uint32_t)b, nodes, n, starts, keys, px, py, pz, g, mark, sol);
        uint32_t start = b ? node_voxels[b - 1] : 0, k = 0;
        for (uint32_t i = 0; i < NVPN; ++i)
            if (mark[i]) { voxel_ids[start + k] = i; solids[start + k] = sol[i]; ++k; }
    }
}

/* ---------------------------------------------------------- P2G / G2P */
static inline void ref_face_offset(int dim, double hs, double* bx, double* by, double* bz) {
    if (dim == 0) { *by += hs; *bz += hs; }
    else if (dim == 1) { *bx += hs; *bz += hs; }
    else { *by += hs; *bx += hs; }
}
/* weightFromDistance (particles.cu:370-377) */
static inline double ref_weight(double d, double R) { return (d > R) ? 0.0 : 1.0 - d / R; }

void orc_ref_p2g(uint32_t nodes, int64_t n, const uint32_t* starts, const uint32_t* keys,
                 const double* px, const double* py, const double* pz, const double* vdim,
                 const uint32_t* node_voxels, const uint32_t* voxel_ids, const int8_t* solids,
                 orc_grid g, int dim, double* voxel_u) {
    double scw = ref_scw(g), hs = scw / 2.0, R = 2.0 * scw;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t bb = 0; bb < (int64_t)nodes; ++bb) {
        uint32_t b = (uint32_t)bb;
        double U[NVPN], W[NVPN];
        int8_t S[NVPN];
        memset(U, 0, sizeof(U));
        memset(W, 0, sizeof(W));   /* the reference leaves this array uninitialised (particles.cu:412-415) */
        memset(S, 0, sizeof(S));
        uint32_t vs = b ? node_voxels[b - 1] : 0, ve = node_voxels[b];
        for (uint32_t k = vs; k < ve; ++k) S[voxel_ids[k]] = solids[k];
        uint32_t last = (b == nodes - 1) ? (uint32_t)n : starts[b + 1];
        for (uint32_t idx = starts[b]; idx < last; ++idx) {
            uint32_t qx, qy, qz;
            ref_decompose(keys[idx], g, &qx, &qy, &qz);
            double lx = ref_local(px[idx], g.negX, qx, g.cellSize, scw);
            double ly = ref_local(py[idx], g.negY, qy, g.cellSize, scw);
            double lz = ref_local(pz[idx], g.negZ, qz, g.cellSize, scw);
            uint32_t sx = sat_u32_d(floor(lx / scw)), sy = sat_u32_d(floor(ly / scw)), sz = sat_u32_d(floor(lz / scw));
            double v = vdim[idx];
            for (int x = (int)(sx - APRON); (uint32_t)x < sx + APRON; ++x)
                for (int y = (int)(sy - APRON); (uint32_t)y < sy + APRON; ++y)
                    for (int z = (int)(sz - APRON); (uint32_t)z < sz + APRON; ++z) {
                        double bx = x * scw, by = y * scw, bz = z * scw;
                        ref_face_offset(dim, hs, &bx, &by, &bz);
                        double w = ref_weight(ref_dist(lx - bx, ly - by, lz - bz), R);
                        if ((uint32_t)x < NV1D && (uint32_t)y < NV1D && (uint32_t)z < NV1D) {
                            uint32_t id = x + y * NV1D + z * NV1D * NV1D;
                            W[id] += w;
                            U[id] += w * v;
                        }
                    }
        }
        for (uint32_t i = 0; i < NVPN; ++i) if (S[i]) U[i] = 0.0;
        for (uint32_t k = vs; k < ve; ++k) voxel_u[k] = U[voxel_ids[k]] / (W[voxel_ids[k]] + 0.0000001);
    }
}

void orc_ref_g2p(uint32_t nodes, int64_t n, const uint32_t* starts, const uint32_t* keys,
                 const double* px, const double* py, const double* pz,
                 const uint32_t* node_voxels, const uint32_t* voxel_ids, const double* voxel_u,
                 orc_grid g, int dim, double* vdim) {
    double scw = ref_scw(g), hs = scw / 2.0, R = 2.0 * scw;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t bb = 0; bb < (int64_t)nodes; ++bb) {
        uint32_t b = (uint32_t)bb;
        double U[NVPN];
        memset(U, 0, sizeof(U));
        uint32_t vs = b ? node_voxels[b - 1] : 0, ve = node_voxels[b];
        for (uint32_t k = vs; k < ve; ++k) U[voxel_ids[k]] = voxel_u[k];
        uint32_t last = (b == nodes - 1) ? (uint32_t)n : starts[b + 1];
        for (uint32_t idx = starts[b]; idx < last; ++idx) {
            uint32_t qx, qy, qz;
            ref_decompose(keys[idx], g, &qx, &qy, &qz);
            double lx = ref_local(px[idx], g.negX, qx, g.cellSize, scw);
            double ly = ref_local(py[idx], g.negY, qy, g.cellSize, scw);
            double lz = ref_local(pz[idx], g.negZ, qz, g.cellSize, scw);
            uint32_t sx = sat_u32_d(floor(lx / scw)), sy = sat_u32_d(floor(ly / scw)), sz = sat_u32_d(floor(lz / scw));
            double vel = 0.0, ws = 0.0;
            for (int x = (int)(sx - APRON); (uint32_t)x < NV1D && (uint32_t)x < sx + APRON; ++x)
                for (int y = (int)(sy - APRON); (uint32_t)y < NV1D && (uint32_t)y < sy + APRON; ++y)
                    for (int z = (int)(sz - APRON); (uint32_t)z < NV1D && (uint32_t)z < sz + APRON; ++z) {
                        double bx = x * scw, by = y * scw, bz = z * scw;
                        ref_face_offset(dim, hs, &bx, &by, &bz);
                        double w = ref_weight(ref_dist(lx - bx, ly - by, lz - bz), R);
                        uint32_t id = x + y * NV1D + z * NV1D * NV1D;
                        if (U[id] != 0.0) {                        /* zero voxels skipped (Q10) */
                            ws += w;
                            vel = fma(w, U[id], vel);
                        }
                    }
            vdim[idx] = vel / (ws + 0.00000001);
        }
    }
}

void orc_ref_advect(int64_t n, double dt, double* pos, const double* v) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) pos[i] = fma(dt, v[i], pos[i]);
}

void orc_ref_move_solids_targets(uint32_t nodes, int64_t n, const uint32_t* starts, const uint32_t* keys,
                                 const double* px, const double* py, const double* pz,
                                 const uint32_t* node_voxels, const uint32_t* voxel_ids, const int8_t* solids,
                                 orc_grid g, uint32_t* new_voxel) {
    double scw = ref_scw(g);
    for (uint32_t b = 0; b < nodes; ++b) {
        int8_t S[NVPN];
        uint32_t proc[NVPN];
        memset(S, 0, sizeof(S));
        for (uint32_t i = 0; i < NVPN; ++i) proc[i] = NVPN;
        uint32_t vs = b ? node_voxels[b - 1] : 0, ve = node_voxels[b];
        for (uint32_t k = vs; k < ve; ++k) { S[voxel_ids[k]] = solids[k]; proc[k - vs] = voxel_ids[k]; }
        uint32_t last = (b == nodes - 1) ? (uint32_t)n : starts[b + 1];
        for (uint32_t idx = starts[b]; idx < last; ++idx) {
            uint32_t qx, qy, qz;
            ref_decompose(keys[idx], g, &qx, &qy, &qz);
            double lx = ref_local(px[idx], g.negX, qx, g.cellSize, scw);
            double ly = ref_local(py[idx], g.negY, qy, g.cellSize, scw);
            double lz = ref_local(pz[idx], g.negZ, qz, g.cellSize, scw);
            uint32_t sx = sat_u32_d(floor(lx / scw)), sy = sat_u32_d(floor(ly / scw)), sz = sat_u32_d(floor(lz / scw));
            new_voxel[idx] = 0xFFFFFFFFu;
            if (sx >= NV1D || sy >= NV1D || sz >= NV1D || S[sx + sy * NV1D + sz * NV1D * NV1D]) {
                /* the reference scans for the first SOLID voxel of the node (Q8),
                 * bounded here by the node's own list */
                uint32_t i = 0;
                while (i < ve - vs && !S[proc[i]]) ++i;
                new_voxel[idx] = (i < NVPN) ? proc[i] : NVPN;
            }
        }
    }
}

/* ----------------------------------------------------------- pressure */
static void getmax_level(int64_t n, const double* a, double* out, int absolute) {
    int64_t nb = n / 512 + 1;
    for (int64_t b = 0; b < nb; ++b) {
        int64_t i0 = b * 512, i1 = b * 512 + 256;
        double s0 = (i0 < n) ? a[i0] : 0.0;
        double s1 = (i1 < n) ? a[i1] : 0.0;
        /* getMaxFromArray compares shared[t] with shared[t+blockDim.x] at every
         * level, so each block returns the pick of its elements 0 and 256 */
        double r;
        if (absolute) r = (fabs(s0) > fabs(s1)) ? s0 : s1;
        else r = (s0 > s1) ? s0 : s1;
        out[b] = r;
    }
}

double orc_ref_getmax(int64_t n, const double* a, int absolute) {
    int64_t nb = n / 512 + 1;
    double* o1 = (double*)malloc(sizeof(double) * (size_t)nb);
    double* o2 = (double*)malloc(sizeof(double) * (size_t)(nb / 512 + 1));
    getmax_level(n, a, o1, absolute);
    for (int64_t i = nb; i > 1; i = i / 512 + 1) {
        getmax_level(i, o1, o2, absolute);
        double* t = o1; o1 = o2; o2 = t;
    }
    double r = o1[0];
    free(o1);
    free(o2);
    return r;
}

void orc_ref_gravity(int64_t nvox, const int8_t* solids, double* uy, double dt, int remove) {
    const double c = (double)(-9.8f);
    for (int64_t i = 0; i < nvox; ++i)
        if (!solids[i]) uy[i] = remove ? fma(-c, dt, uy[i]) : fma(c, dt, uy[i]);
}

static void ref_neighbor_apron(uint32_t nid, const uint32_t* node_voxels, const uint32_t* voxel_ids,
                               const double* data, double* S, int xo, int yo, int zo) {
    uint32_t vs = nid ? node_voxels[nid - 1] : 0, ve = node_voxels[nid];
    for (uint32_t k = vs; k < ve; ++k) {
        uint32_t id = voxel_ids[k];
        uint32_t sx = id % NV1D, sy = (id % 64u) / NV1D, sz = id / 64u;
        uint32_t tx = sx, ty = sy, tz = sz;
        if (xo < 0) { if (sx >= NV1D + (uint32_t)xo) { tx = sx - NV1D - (uint32_t)xo; S[tx + ty * 8 + tz * 64] += data[k]; } }
        else if (xo > 0) { if (sx < (uint32_t)xo) { tx = NV1D - (uint32_t)xo + sx; S[tx + ty * 8 + tz * 64] += data[k]; } }
        else if (yo < 0) { if (sy >= NV1D + (uint32_t)yo) { ty = sy - NV1D - (uint32_t)yo; S[tx + ty * 8 + tz * 64] += data[k]; } }
        else if (yo > 0) { if (sy < (uint32_t)yo) { ty = NV1D - (uint32_t)yo + sy; S[tx + ty * 8 + tz * 64] += data[k]; } }
        else if (zo < 0) { if (sz >= NV1D + (uint32_t)zo) { tz = sz - NV1D - (uint32_t)zo; S[tz + ty * 8 + tz * 64] += data[k]; } } /* Q6 */
        else if (zo > 0) { if (sz < (uint32_t)zo) { tz = NV1D - (uint32_t)zo + sz; S[tx + ty * 8 + tz * 64] += data[k]; } }
    }
}

void orc_ref_divergence(uint32_t nodes, const uint32_t* node_voxels, const uint32_t* voxel_ids,
                        const double* ux, const double* uy, const double* uz, orc_grid g,
                        const uint32_t* ytable, const uint32_t* starts, const uint32_t* keys, double* divU) {
    int64_t nvox = nodes ? node_voxels[nodes - 1] : 0;
    memset(divU, 0, sizeof(double) * (size_t)nvox);
    const double* data[3] = {ux, uy, uz};
    for (int dim = 0; dim < 3; ++dim) {
#pragma omp parallel for schedule(dynamic, 16)
        for (int64_t bb = 0; bb < (int64_t)nodes; ++bb) {
            uint32_t b = (uint32_t)bb;
            double S[NVPN];
            memset(S, 0, sizeof(S));
            uint32_t vs = b ? node_voxels[b - 1] : 0, ve = node_voxels[b];
            for (uint32_t k = vs; k < ve; ++k) S[voxel_ids[k]] += data[dim][k];
            uint32_t cur = keys[starts[b]];
            uint32_t cx = cur % g.sizeX, cy = (cur % (g.sizeX * g.sizeY)) / g.sizeX, cz = cur / (g.sizeX * g.sizeY);
            int xl = (int)(cx - 1), xr = (int)(cx + 1), yl = (int)(cy - 1), yr = (int)(cy + 1), zl = (int)(cz - 1), zr = (int)(cz + 1);
            const int T = 4;                                   /* 2 * numApronCells */
            uint32_t nid;
            if (xl >= 0 && b > 0)
                if (keys[starts[b - 1]] == cur - 1) ref_neighbor_apron(b - 1, node_voxels, voxel_ids, data[dim], S, -T, 0, 0);
            if ((uint32_t)xr < g.sizeX && b < nodes - 1)
                if (keys[starts[b + 1]] == cur + 1) ref_neighbor_apron(b + 1, node_voxels, voxel_ids, data[dim], S, T, 0, 0);
            if (yl >= 0 && (nid = ytable[(uint32_t)yl + cz * g.sizeY]) < nodes)
                ref_neighbor_apron(nid, node_voxels, voxel_ids, data[dim], S, 0, -T, 0);
            if ((uint32_t)yr < g.sizeY && (nid = ytable[(uint32_t)yr + cz * g.sizeY]) < nodes)
                ref_neighbor_apron(nid, node_voxels, voxel_ids, data[dim], S, 0, T, 0);
            if (zl >= 0 && (nid = ytable[(uint32_t)zl * g.sizeY + cy]) < nodes)
                ref_neighbor_apron(nid, node_voxels, voxel_ids, data[dim], S, 0, 0, -T);
            if ((uint32_t)zr < g.sizeZ && (nid = ytable[(uint32_t)zr * g.sizeY + cy]) < nodes)
                ref_neighbor_apron(nid, node_voxels, voxel_ids, data[dim], S, 0, 0, T);
            for (uint32_t k = vs; k < ve; ++k) {
                uint32_t id = voxel_ids[k];
                double d = 0.0;
                if (dim == 0) { if (id % 8 < 7) d = S[id + 1] - S[id]; }
                else if (dim == 1) { if ((id % 64) / 8 < 7) d = S[id + 8] - S[id]; }
                else { if (id / 64 < 7) d = S[id + 64] - S[id]; }
                divU[k] += d;
            }
        }
    }
}

/* isApronCell (voxelSolveFunctions.cu:275-284): y is computed with the same
 * precedence slip as the activation kernel, so it equals x. */
static inline int ref_is_apron(uint32_t id) {
    uint32_t x = id % NV1D, y = (id % NV1D * NV1D) / NV1D, z = id / (NV1D * NV1D);
    return x < 1 || x >= 7 || y < 1 || y >= 7 || z < 1 || z >= 7;
}
static inline int ref_is_red(uint32_t id) {
    uint32_t x = id % NV1D, y = (id % 64u) / NV1D, z = id / 64u;
    return !((x + y + z) & 1u);
}

void orc_ref_gs_pass(uint32_t nodes, const uint32_t* node_voxels, const uint32_t* voxel_ids,
                     const int8_t* solids, const double* divU, double* p, double* res,
                     double density, double dt, orc_grid g, int red, double w) {
    double vsz = ref_scw(g);
    double scale = dt / (density * vsz * vsz);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t bb = 0; bb < (int64_t)nodes; ++bb) {
        uint32_t b = (uint32_t)bb;
        double D[NVPN], P[NVPN], Rr[NVPN];
        int8_t S[NVPN];
        memset(D, 0, sizeof(D)); memset(P, 0, sizeof(P)); memset(Rr, 0, sizeof(Rr)); memset(S, 0, sizeof(S));
        uint32_t vs = b ? node_voxels[b - 1] : 0, ve = node_voxels[b];
        for (uint32_t k = vs; k < ve; ++k) { uint32_t id = voxel_ids[k]; D[id] = divU[k]; P[id] = p[k]; S[id] = solids[k]; }
        for (uint32_t k = vs; k < ve; ++k) {
            uint32_t v = voxel_ids[k];
            if ((red == ref_is_red(v)) && !S[v] && !ref_is_apron(v)) {
                double Ad = 0.0, Anx = 0.0, Apx = 0.0, Any = 0.0, Apy = 0.0, Anz = 0.0, Apz = 0.0;
                if (!S[v - 1]) { if (D[v - 1] != 0.0) Anx = -scale; Ad += scale; }
                if (!S[v + 1]) { if (D[v + 1] != 0.0) Apx = -scale; Ad += scale; }
                if (!S[v - 8]) { if (D[v - 8] != 0.0) Any = -scale; Ad += scale; }
                if (!S[v + 8]) { if (D[v + 8] != 0.0) Apy = -scale; Ad += scale; }
                if (!S[v - 64]) { if (D[v - 64] != 0.0) Anz = -scale; Ad += scale; }
                if (!S[v + 64]) { if (D[v + 64] != 0.0) Apz = -scale; Ad += scale; }
                double s = Anx * P[v - 1];
                s = fma(Apx, P[v + 1], s);
                s = fma(Any, P[v - 8], s);
                s = fma(Apy, P[v + 8], s);
                s = fma(Anz, P[v - 64], s);
                s = fma(Apz, P[v + 64], s);
                double Adg = Ad + 0.000000001;
                double t = (-D[v] - s) / Adg - P[v];
                P[v] = fma(w, t, P[v]);
                Rr[v] = fma(-Adg, P[v], -D[v]) + s;
            }
        }
        for (uint32_t k = vs; k < ve; ++k) { uint32_t id = voxel_ids[k]; p[k] = P[id]; res[k] = Rr[id]; }
    }
}

double orc_ref_gs_solve(uint32_t nodes, const uint32_t* node_voxels, const uint32_t* voxel_ids,
                        const int8_t* solids, const double* divU, double* p, double* res,
                        double density, double dt, orc_grid g, double threshold, uint32_t max_iter,
                        uint32_t* iters) {
    double maxR = 10.0, prevR = 100.0;
    uint32_t it = 0;
    int64_t nvox = nodes ? node_voxels[nodes - 1] : 0;
    const double w = 1.9;
    while (maxR > threshold && it < max_iter) {
        orc_ref_gs_pass(nodes, node_voxels, voxel_ids, solids, divU, p, res, density, dt, g, 1, w);
        orc_ref_gs_pass(nodes, node_voxels, voxel_ids, solids, divU, p, res, density, dt, g, 0, w);
        if (it % 1024 == 0) { prevR = maxR; maxR = orc_ref_getmax(nvox, res, 1); }
        ++it;
        if (it == max_iter || (fabs(prevR - maxR) < threshold / 1000 && maxR > threshold)) break;
    }
    if (iters) *iters = it;
    return maxR;
}

void orc_ref_velocity_update(uint32_t nodes, const uint32_t* node_voxels, const uint32_t* voxel_ids,
                             const int8_t* solids, const double* p, double* ux, double* uy, double* uz,
                             double dt, double density, orc_grid g) {
    double vsz = ref_scw(g);
    double scale = dt / (density * vsz * vsz);
    double* U3[3] = {ux, uy, uz};
    const uint32_t stride[3] = {1, 8, 64};
    for (int dim = 0; dim < 3; ++dim) {
#pragma omp parallel for schedule(dynamic, 16)
        for (int64_t bb = 0; bb < (int64_t)nodes; ++bb) {
            uint32_t b = (uint32_t)bb;
            double P[NVPN], U[NVPN];
            int8_t S[NVPN];
            memset(P, 0, sizeof(P)); memset(U, 0, sizeof(U)); memset(S, 0, sizeof(S));
            uint32_t vs = b ? node_voxels[b - 1] : 0, ve = node_voxels[b];
            for (uint32_t k = vs; k < ve; ++k) { uint32_t id = voxel_ids[k]; U[id] = U3[dim][k]; P[id] = p[k]; S[id] = solids[k]; }
            for (uint32_t k = vs; k < ve; ++k) {
                uint32_t v = voxel_ids[k];
                if (!S[v] && !ref_is_apron(v)) {
                    double dp = 0.0;
                    if (!S[v - stride[dim]]) dp = P[v] - P[v - stride[dim]];
                    U[v] = fma(-dp, scale, U[v]);
                }
            }
            for (uint32_t k = vs; k < ve; ++k) U3[dim][k] = U[voxel_ids[k]];
        }
    }
}

int orc_ref_substep(int64_t n, double* px, double* py, double* pz, double* vx, double* vy, double* vz,
                    orc_grid g, double frameDt, double elapsedThisFrame, int permute_velocities,
                    orc_ref_step_info* info) {
    if (n <= 0) return -1;
    size_t N = (size_t)n;
    uint32_t* keys = (uint32_t*)malloc(4 * N);
    uint32_t* skeys = (uint32_t*)malloc(4 * N);
    uint32_t* perm = (uint32_t*)malloc(4 * N);
    uint32_t* fs = (uint32_t*)malloc(4 * N);
    double* tmp = (double*)malloc(8 * N);
    /* initialize(): alignParticlesToGrid, sortParticles, generateVoxels (particles.cu:805-812) */
    orc_ref_keys(n, px, py, pz, g, keys);
    orc_sort_pairs(n, keys, skeys, perm);
    double* arrs[6] = {px, py, pz, vx, vy, vz};
    int nperm = permute_velocities ? 6 : 3;
    for (int a = 0; a < nperm; ++a) { orc_gather_f64(n, perm, arrs[a], tmp); memcpy(arrs[a], tmp, 8 * N); }
    uint32_t nodes = orc_mark_unique_scan(n, skeys, fs);
    uint32_t* starts = (uint32_t*)malloc(4 * (size_t)nodes);
    orc_cell_starts(n, fs, starts);
    uint32_t* ytab = (uint32_t*)malloc(4 * (size_t)g.sizeY * g.sizeZ);
    orc_ydim_rows(nodes, starts, skeys, g, ytab);
    uint32_t* nv = (uint32_t*)malloc(4 * (size_t)nodes);
    orc_ref_voxel_counts(nodes, n, starts, skeys, px, py, pz, g, nv);
    orc_inclusive_scan(nodes, nv);
    uint32_t nvox = nv[nodes - 1];
    uint32_t* ids = (uint32_t*)malloc(4 * (size_t)nvox);
    int8_t* sol = (int8_t*)malloc((size_t)nvox);
    orc_ref_voxel_ids(nodes, n, starts, skeys, px, py, pz, g, nv, ids, sol);
    double* U[3];
    for (int d = 0; d < 3; ++d) U[d] = (double*)malloc(8 * (size_t)nvox);
    double* divU = (double*)malloc(8 * (size_t)nvox);
    double* p = (double*)calloc(nvox, 8);
    double* res = (double*)calloc(nvox, 8);
    /* particleVelToVoxels */
    double* vel[3] = {vx, vy, vz};
    for (int d = 0; d < 3; ++d) orc_ref_p2g(nodes, n, starts, skeys, px, py, pz, vel[d], nv, ids, sol, g, d, U[d]);
    /* pressureSolve (particles.cu:507-555) */
    const double density = 0.014, threshold = 0.01;
    double vmax = fmax(fabs(orc_ref_getmax(n, vx, 1)), fmax(fabs(orc_ref_getmax(n, vy, 1)), fabs(orc_ref_getmax(n, vz, 1))));
    double voxelSize = (double)g.cellSize / (8.0 - 2.0 * 2.0);
    double dt = 0.7 * (voxelSize / vmax);
    if (frameDt - elapsedThisFrame < dt) dt = frameDt - elapsedThisFrame;
    orc_ref_gravity(nvox, sol, U[1], dt, 0);
    orc_ref_divergence(nodes, nv, ids, U[0], U[1], U[2], g, ytab, starts, skeys, divU);
    double prevTerm = 100.0, term;
    uint32_t it = 0, total_it = 0;
    while (prevTerm - (term = orc_ref_gs_solve(nodes, nv, ids, sol, divU, p, res, density, dt, g, threshold, 16384, &it)) > 0) {
        total_it += it;
        if (term < threshold) break;
        orc_ref_gravity(nvox, sol, U[1], dt, 1);
        dt /= 2.0;
        memset(p, 0, 8 * (size_t)nvox);
        orc_ref_gravity(nvox, sol, U[1], dt, 0);
        prevTerm = term;
        orc_ref_divergence(nodes, nv, ids, U[0], U[1], U[2], g, ytab, starts, skeys, divU);
        it = 0;
    }
    total_it += it;
    /* updateVoxelVelocities, voxelVelsToParticles, advectParticles */
    orc_ref_velocity_update(nodes, nv, ids, sol, p, U[0], U[1], U[2], dt, density, g);
    for (int d = 0; d < 3; ++d) orc_ref_g2p(nodes, n, starts, skeys, px, py, pz, nv, ids, U[d], g, d, vel[d]);
    orc_ref_advect(n, dt, px, vx);
    orc_ref_advect(n, dt, py, vy);
    orc_ref_advect(n, dt, pz, vz);
    if (info) { info->nodes = nodes; info->voxels = nvox; info->gs_iters_total = total_it; info->dt = dt; info->residual = term; }
    for (int d = 0; d < 3; ++d) free(U[d]);
    free(keys); free(skeys); free(perm); free(fs); free(tmp); free(starts); free(ytab); free(nv);
    free(ids); free(sol); free(divU); free(p); free(res);
    return 0;
}

/* =========================================== native-mode step (FP64) ====
 * Staggered MAC grid of nx*ny*nz cells of size h.  Face (i,j,k) of a
 * component is the negative face of cell (i,j,k); the positive domain wall
 * faces (i == nx) are not stored and read as 0.  Cell types: 0 air, 1 fluid,
 * 2 solid; the exterior of the box is solid. */
#define NAT_AIR 0
#define NAT_FLUID 1
#define NAT_SOLID 2

static inline int64_t nat_idx(const orc_nat_params* P, int i, int j, int k) {
    return (int64_t)i + (int64_t)P->nx * ((int64_t)j + (int64_t)P->ny * k);
}
/* cell index of a float position, in float arithmetic as the device does */
static inline int nat_cell(float p, float o, float h, int n) {
    float t = floorf((p - o) / h);
    int c = (t >= (float)n) ? n - 1 : (int)t;
    if (!(t > 0.0f)) c = 0;
    return c;
}

void orc_nat_keys(int64_t n, const float* pos, const orc_nat_params* P, uint32_t* keys) {
    float ox = (float)P->ox, oy = (float)P->oy, oz = (float)P->oz, h = (float)P->h;
    int tx = P->nx / 8, ty = P->ny / 8;
    for (int64_t p = 0; p < n; ++p) {
        int i = nat_cell(pos[3 * p], ox, h, P->nx), j = nat_cell(pos[3 * p + 1], oy, h, P->ny), k = nat_cell(pos[3 * p + 2], oz, h, P->nz);
        keys[p] = (uint32_t)((i >> 3) + tx * ((j >> 3) + ty * (k >> 3)));
    }
}

/* axis sample: clamp s to [0, M], base in [0, M-1] */
static inline void nat_axis(double s, int M, int* i0, double* f) {
    if (s < 0.0) s = 0.0;
    if (s > (double)M) s = (double)M;
    int b = (int)floor(s);
    if (b > M - 1) b = M - 1;
    if (b < 0) b = 0;
    *i0 = b;
    *f = s - (double)b;
}

/* component c: node ranges M = (nx, ny-1, nz-1) for u, etc.; sample offsets */
static void nat_stencil(const orc_nat_params* P, int c, double gx, double gy, double gz,
                        int* i0, int* j0, int* k0, double* fx, double* fy, double* fz) {
    double sx = gx - (c == 0 ? 0.0 : 0.5), sy = gy - (c == 1 ? 0.0 : 0.5), sz = gz - (c == 2 ? 0.0 : 0.5);
    nat_axis(sx, c == 0 ? P->nx : P->nx - 1, i0, fx);
    nat_axis(sy, c == 1 ? P->ny : P->ny - 1, j0, fy);
    nat_axis(sz, c == 2 ? P->nz : P->nz - 1, k0, fz);
}
static inline int nat_wall(const orc_nat_params* P, int c, int i, int j, int k) {
    if (c == 0) return i == 0 || i == P->nx;
    if (c == 1) return j == 0 || j == P->ny;
    return k == 0 || k == P->nz;
}

/* P2G of one particle into the face sums (wall faces skipped) */
static void nat_p2g_particle(const orc_nat_params* P, int64_t nc, const float* pos, const float* vel, int64_t p,
                             double* const* comp, double* wt) {
    double gx = ((double)pos[3 * p] - P->ox) / P->h;
    double gy = ((double)pos[3 * p + 1] - P->oy) / P->h;
    double gz = ((double)pos[3 * p + 2] - P->oz) / P->h;
    for (int c = 0; c < 3; ++c) {
        int i0, j0, k0;
        double fx, fy, fz;
        nat_stencil(P, c, gx, gy, gz, &i0, &j0, &k0, &fx, &fy, &fz);
        for (int dk = 0; dk < 2; ++dk)
            for (int dj = 0; dj < 2; ++dj)
                for (int di = 0; di < 2; ++di) {
                    int i = i0 + di, j = j0 + dj, k = k0 + dk;
                    if (nat_wall(P, c, i, j, k)) continue;
                    double ww = (di ? fx : 1.0 - fx) * (dj ? fy : 1.0 - fy) * (dk ? fz : 1.0 - fz);
                    int64_t id = nat_idx(P, i, j, k);
                    comp[c][id] += ww * (double)vel[3 * p + c];
                    wt[(int64_t)c * nc + id] += ww;
                }
    }
}

/* Trilinear P2G onto the staggered faces, sums in FP64.  Particles are
 * bucketed by 8-cell slabs of z; a particle of slab s touches nodes of z in
 * [8s-1, 8s+8] only, so slabs two apart never share a node: the even slabs
 * run in parallel, then the odd ones.  Within a slab particles keep their
 * input order, so the result does not depend on the thread count. */
void orc_nat_p2g(int64_t n, const float* pos, const float* vel, const orc_nat_params* P,
                 double* u, double* v, double* w, uint8_t* fluid) {
    int64_t nc = (int64_t)P->nx * P->ny * P->nz;
    double* comp[3] = {u, v, w};
    double* wt = (double*)calloc((size_t)nc * 3, sizeof(double));
    for (int c = 0; c < 3; ++c) memset(comp[c], 0, sizeof(double) * (size_t)nc);
    if (fluid) memset(fluid, 0, (size_t)nc);
    float fox = (float)P->ox, foy = (float)P->oy, foz = (float)P->oz, fh = (float)P->h;
    const int nslab = (P->nz + 7) / 8;
    int64_t* cnt = (int64_t*)calloc((size_t)nslab + 1, sizeof(int64_t));
    int* slab = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int64_t p = 0; p < n; ++p) {
        int kc = nat_cell(pos[3 * p + 2], foz, fh, P->nz);
        slab[p] = kc / 8;
        cnt[slab[p] + 1]++;
        if (fluid) fluid[nat_idx(P, nat_cell(pos[3 * p], fox, fh, P->nx), nat_cell(pos[3 * p + 1], foy, fh, P->ny), kc)] = 1;
    }
    for (int s2 = 0; s2 < nslab; ++s2) cnt[s2 + 1] += cnt[s2];
    int64_t* order = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)nslab);
    memcpy(fill, cnt, sizeof(int64_t) * (size_t)nslab);
    for (int64_t p = 0; p < n; ++p) order[fill[slab[p]]++] = p;
    for (int phase = 0; phase < 2; ++phase) {
#pragma omp parallel for schedule(dynamic, 1)
        for (int sl = phase; sl < nslab; sl += 2)
            for (int64_t q = cnt[sl]; q < cnt[sl + 1]; ++q) nat_p2g_particle(P, nc, pos, vel, order[q], comp, wt);
    }
    free(cnt); free(slab); free(order); free(fill);
#pragma omp parallel for schedule(static)
    for (int64_t id = 0; id < nc; ++id)
        for (int c = 0; c < 3; ++c) {
            double ww = wt[(int64_t)c * nc + id];
            comp[c][id] = ww > 0.0 ? comp[c][id] / ww : 0.0;
        }
    free(wt);
}

static inline int nat_type(const orc_nat_params* P, const uint8_t* type, int i, int j, int k) {
    if (i < 0 || j < 0 || k < 0 || i >= P->nx || j >= P->ny || k >= P->nz) return NAT_SOLID;
    return type[nat_idx(P, i, j, k)];
}

void orc_nat_apply_A(const uint8_t* type, const double* x, double* y, const orc_nat_params* P) {
    static const int off[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
#pragma omp parallel for schedule(static)
    for (int k = 0; k < P->nz; ++k)
        for (int j = 0; j < P->ny; ++j)
            for (int i = 0; i < P->nx; ++i) {
                int64_t id = nat_idx(P, i, j, k);
                if (type[id] != NAT_FLUID) { y[id] = 0.0; continue; }
                double d = 0.0, s = 0.0;
                for (int q = 0; q < 6; ++q) {
                    int t = nat_type(P, type, i + off[q][0], j + off[q][1], k + off[q][2]);
                    if (t == NAT_SOLID) continue;
                    d += 1.0;
                    if (t == NAT_FLUID) s += x[nat_idx(P, i + off[q][0], j + off[q][1], k + off[q][2])];
                }
                y[id] = d * x[id] - s;
            }
}

static double nat_dot(int64_t nc, const double* a, const double* b) {
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (int64_t i = 0; i < nc; ++i) s += a[i] * b[i];
    return s;
}

/* Jacobi-PCG over the fluid cells, FP64 throughout.  The work runs on the
 * list of fluid cells (OpenMP); dot products are OpenMP reductions. */
int orc_nat_pcg(const uint8_t* type, const double* b, double* x, const orc_nat_params* P, double* rel_res) {
    static const int off[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    int64_t nc = (int64_t)P->nx * P->ny * P->nz;
    int64_t nf = 0;
    for (int64_t i = 0; i < nc; ++i) nf += (type[i] == NAT_FLUID);
    int64_t* fl = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nf > 0 ? nf : 1));
    /* neighbour slots of each fluid cell: -1 solid (no coupling), -2 air (Dirichlet 0) */
    int64_t* nb = (int64_t*)malloc(sizeof(int64_t) * 6 * (size_t)(nf > 0 ? nf : 1));
    double* r = (double*)calloc((size_t)nc, 8);
    double* z = (double*)calloc((size_t)nc, 8);
    double* p = (double*)calloc((size_t)nc, 8);
    double* q = (double*)calloc((size_t)nc, 8);
    double* dinv = (double*)calloc((size_t)nc, 8);
    {
        int64_t f = 0;
        for (int k = 0; k < P->nz; ++k)
            for (int j = 0; j < P->ny; ++j)
                for (int i = 0; i < P->nx; ++i) {
                    int64_t id = nat_idx(P, i, j, k);
                    if (type[id] != NAT_FLUID) continue;
                    int d = 0;
                    for (int s = 0; s < 6; ++s) {
                        int ii = i + off[s][0], jj = j + off[s][1], kk = k + off[s][2];
                        int t = nat_type(P, type, ii, jj, kk);
                        if (t != NAT_SOLID) ++d;
                        nb[6 * f + s] = (t == NAT_SOLID) ? -1 : (t == NAT_FLUID ? nat_idx(P, ii, jj, kk) : -2);
                    }
                    dinv[id] = d ? 1.0 / d : 0.0;
                    fl[f++] = id;
                }
    }
#define PCG_FOR _Pragma("omp parallel for schedule(static)") for (int64_t f = 0; f < nf; ++f)
    double bb = 0.0;
#pragma omp parallel for reduction(+ : bb) schedule(static)
    for (int64_t f = 0; f < nf; ++f) { int64_t id = fl[f]; bb += b[id] * b[id]; }
    PCG_FOR { int64_t id = fl[f]; r[id] = b[id]; z[id] = r[id] * dinv[id]; p[id] = z[id]; }
    for (int64_t i = 0; i < nc; ++i) x[i] = 0.0;
    double bn = sqrt(bb);
    double rz = 0.0;
#pragma omp parallel for reduction(+ : rz) schedule(static)
    for (int64_t f = 0; f < nf; ++f) { int64_t id = fl[f]; rz += r[id] * z[id]; }
    int it = 0;
    if (bn > 0.0) {
        for (it = 1; it <= P->max_iter; ++it) {
            double pq = 0.0;
#pragma omp parallel for reduction(+ : pq) schedule(static)
            for (int64_t f = 0; f < nf; ++f) {
                int64_t id = fl[f];
                double d = 0.0, sn = 0.0;
                for (int s = 0; s < 6; ++s) {
                    int64_t m = nb[6 * f + s];
                    if (m == -1) continue;
                    d += 1.0;
                    if (m >= 0) sn += p[m];
                }
                q[id] = d * p[id] - sn;
                pq += p[id] * q[id];
            }
            double alpha = rz / pq;
            double rr = 0.0;
#pragma omp parallel for reduction(+ : rr) schedule(static)
            for (int64_t f = 0; f < nf; ++f) {
                int64_t id = fl[f];
                x[id] += alpha * p[id];
                r[id] -= alpha * q[id];
                rr += r[id] * r[id];
            }
            if (sqrt(rr) <= P->tol * bn) break;
            double rzn = 0.0;
#pragma omp parallel for reduction(+ : rzn) schedule(static)
            for (int64_t f = 0; f < nf; ++f) {
                int64_t id = fl[f];
                z[id] = r[id] * dinv[id];
                rzn += r[id] * z[id];
            }
            double beta = rzn / rz;
            rz = rzn;
            PCG_FOR { int64_t id = fl[f]; p[id] = z[id] + beta * p[id]; }
        }
        if (it > P->max_iter) it = P->max_iter;
    }
#undef PCG_FOR
    if (rel_res) {
        orc_nat_apply_A(type, x, q, P);
        double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
        for (int64_t f = 0; f < nf; ++f) { int64_t id = fl[f]; double e = b[id] - q[id]; s += e * e; }
        *rel_res = bn > 0.0 ? sqrt(s) / bn : 0.0;
    }
    free(r); free(z); free(p); free(q); free(dinv); free(fl); free(nb);
    return it;
}

/* trilinear sample of a face grid (wall faces read 0) */
static double nat_sample(const orc_nat_params* P, const double* f, int c, double gx, double gy, double gz) {
    int i0, j0, k0;
    double fx, fy, fz, s = 0.0;
    nat_stencil(P, c, gx, gy, gz, &i0, &j0, &k0, &fx, &fy, &fz);
    for (int dk = 0; dk < 2; ++dk)
        for (int dj = 0; dj < 2; ++dj)
            for (int di = 0; di < 2; ++di) {
                int i = i0 + di, j = j0 + dj, k = k0 + dk;
                if (nat_wall(P, c, i, j, k)) continue;
                double ww = (di ? fx : 1.0 - fx) * (dj ? fy : 1.0 - fy) * (dk ? fz : 1.0 - fz);
                s += ww * f[nat_idx(P, i, j, k)];
            }
    return s;
}

int orc_nat_step(int64_t n, float* pos, float* vel, const uint8_t* solid, const orc_nat_params* P,
                 double* u_p2g, double* v_p2g, double* w_p2g, double* phi, orc_nat_info* info) {
    return orc_nat_step_ex(n, pos, vel, solid, P, u_p2g, v_p2g, w_p2g, phi, NULL, NULL, NULL, info);
}

int orc_nat_step_ex(int64_t n, float* pos, float* vel, const uint8_t* solid, const orc_nat_params* P,
                    double* u_p2g, double* v_p2g, double* w_p2g, double* phi, double* u_proj, double* v_proj,
                    double* w_proj, orc_nat_info* info) {
    int64_t nc = (int64_t)P->nx * P->ny * P->nz;
    double* U[3];
    double* Uo[3];
    for (int c = 0; c < 3; ++c) { U[c] = (double*)malloc(8 * (size_t)nc); Uo[c] = (double*)malloc(8 * (size_t)nc); }
    uint8_t* type = (uint8_t*)malloc((size_t)nc);
    double* b = (double*)calloc((size_t)nc, 8);
    double* x = (double*)calloc((size_t)nc, 8);
    orc_nat_p2g(n, pos, vel, P, U[0], U[1], U[2], type);
    int64_t nfluid = 0;
    for (int64_t i = 0; i < nc; ++i) {
        if (solid && solid[i]) type[i] = NAT_SOLID;
        nfluid += (type[i] == NAT_FLUID);
    }
    if (u_p2g) memcpy(u_p2g, U[0], 8 * (size_t)nc);
    if (v_p2g) memcpy(v_p2g, U[1], 8 * (size_t)nc);
    if (w_p2g) memcpy(w_p2g, U[2], 8 * (size_t)nc);
    for (int c = 0; c < 3; ++c) memcpy(Uo[c], U[c], 8 * (size_t)nc);
    /* face classification: wall faces and faces between two solid cells 0,
     * faces between a solid and a non-solid cell the solid velocity, faces
     * touching fluid get gravity */
    const double us[3] = {P->solid_u, P->solid_v, P->solid_w};
    for (int c = 0; c < 3; ++c)
#pragma omp parallel for schedule(static)
        for (int k = 0; k < P->nz; ++k)
            for (int j = 0; j < P->ny; ++j)
                for (int i = 0; i < P->nx; ++i) {
                    int64_t id = nat_idx(P, i, j, k);
                    int ia = i - (c == 0), ja = j - (c == 1), ka = k - (c == 2);
                    int tb = nat_type(P, type, i, j, k), ta = nat_type(P, type, ia, ja, ka);
                    const int wall = ia < 0 || ja < 0 || ka < 0;
                    if (ta == NAT_SOLID || tb == NAT_SOLID) {
                        U[c][id] = (!wall && (ta == NAT_SOLID) != (tb == NAT_SOLID)) ? (double)(float)us[c] : 0.0;
                        continue;
                    }
                    if (c == 1 && (ta == NAT_FLUID || tb == NAT_FLUID)) U[c][id] += P->gravity_y * P->dt;
                }
    /* divergence -> b = -div on fluid cells */
#pragma omp parallel for schedule(static)
    for (int k = 0; k < P->nz; ++k)
        for (int j = 0; j < P->ny; ++j)
            for (int i = 0; i < P->nx; ++i) {
                int64_t id = nat_idx(P, i, j, k);
                if (type[id] != NAT_FLUID) continue;
                double up = (i + 1 < P->nx) ? U[0][nat_idx(P, i + 1, j, k)] : 0.0;
                double vp = (j + 1 < P->ny) ? U[1][nat_idx(P, i, j + 1, k)] : 0.0;
                double wp = (k + 1 < P->nz) ? U[2][nat_idx(P, i, j, k + 1)] : 0.0;
                double div = (up - U[0][id]) + (vp - U[1][id]) + (wp - U[2][id]);
                b[id] = -div;
            }
    double rel = 0.0;
    int it = orc_nat_pcg(type, b, x, P, &rel);
    if (phi) memcpy(phi, x, 8 * (size_t)nc);
    /* projection of fluid-adjacent faces */
    for (int c = 0; c < 3; ++c)
#pragma omp parallel for schedule(static)
        for (int k = 0; k < P->nz; ++k)
            for (int j = 0; j < P->ny; ++j)
                for (int i = 0; i < P->nx; ++i) {
                    int64_t id = nat_idx(P, i, j, k);
                    int ia = i - (c == 0), ja = j - (c == 1), ka = k - (c == 2);
                    int tb = nat_type(P, type, i, j, k), ta = nat_type(P, type, ia, ja, ka);
                    if (ta == NAT_SOLID || tb == NAT_SOLID) continue;
                    if (ta != NAT_FLUID && tb != NAT_FLUID) continue;
                    double pb = (tb == NAT_FLUID) ? x[id] : 0.0;
                    double pa = (ta == NAT_FLUID) ? x[nat_idx(P, ia, ja, ka)] : 0.0;
                    U[c][id] -= pb - pa;
                }
    if (u_proj) memcpy(u_proj, U[0], 8 * (size_t)nc);
    if (v_proj) memcpy(v_proj, U[1], 8 * (size_t)nc);
    if (w_proj) memcpy(w_proj, U[2], 8 * (size_t)nc);
    /* G2P: FLIP blend, then RK2 through the grid velocity; clamp into the box */
    double lo[3] = {P->ox, P->oy, P->oz};
    double hi[3] = {P->ox + P->nx * P->h, P->oy + P->ny * P->h, P->oz + P->nz * P->h};
    double eps = 1e-3 * P->h;
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < n; ++p) {
        double g0[3] = {((double)pos[3 * p] - P->ox) / P->h, ((double)pos[3 * p + 1] - P->oy) / P->h, ((double)pos[3 * p + 2] - P->oz) / P->h};
        double un[3];
        for (int c = 0; c < 3; ++c) {
            un[c] = nat_sample(P, U[c], c, g0[0], g0[1], g0[2]);
            double uo = nat_sample(P, Uo[c], c, g0[0], g0[1], g0[2]);
            double vf = (double)vel[3 * p + c] + (un[c] - uo);
            vel[3 * p + c] = (float)(P->flip * vf + (1.0 - P->flip) * un[c]);
        }
        double xm[3], gm[3];
        for (int c = 0; c < 3; ++c) { xm[c] = (double)pos[3 * p + c] + 0.5 * P->dt * un[c]; gm[c] = (xm[c] - lo[c]) / P->h; }
        float xf[3];
        for (int c = 0; c < 3; ++c) {
            double um = nat_sample(P, U[c], c, gm[0], gm[1], gm[2]);
            double xn = (double)pos[3 * p + c] + P->dt * um;
            if (xn < lo[c] + eps) xn = lo[c] + eps;
            if (xn > hi[c] - eps) xn = hi[c] - eps;
            xf[c] = (float)xn;
        }
        /* a particle that moved into an interior solid cell stays where it
         * started the step and takes the solid's velocity */
        if (solid && solid[nat_idx(P, nat_cell(xf[0], (float)P->ox, (float)P->h, P->nx),
                                   nat_cell(xf[1], (float)P->oy, (float)P->h, P->ny),
                                   nat_cell(xf[2], (float)P->oz, (float)P->h, P->nz))]) {
            for (int c = 0; c < 3; ++c) vel[3 * p + c] = (float)us[c];
        } else {
            for (int c = 0; c < 3; ++c) pos[3 * p + c] = xf[c];
        }
    }
    if (info) { info->iters = it; info->rel_residual = rel; info->fluid_cells = nfluid; }
    for (int c = 0; c < 3; ++c) { free(U[c]); free(Uo[c]); }
    free(type); free(b); free(x);
    return 0;
}

/* ============================================ learned preconditioner (CPU)
 * The product's pressure-preconditioner network, restated for the parity
 * tests (it has no reference counterpart).  Grids are x fastest, nx*ny*nz.
 * f: four 3^3 convolutions, channels 3 -> 16 -> 16 -> 16 -> 1, dilations
 * dil[], ReLU after the first three, zero padding outside the box.  Weights
 * are [27 taps][Cin][Cout] per layer with tap = 9 (dz+1) + 3 (dy+1) + (dx+1)
 * and the neighbour at (i + dil dx, j + dil dy, k + dil dz).  Inputs at a
 * cell: r/s (fluid only), fluid flag, solid flag with s = rms of r over the
 * fluid cells.  The network is N(r) = s (f(r/s) - f(0)) on fluid cells and 0
 * elsewhere; f(0) sees the geometry channels alone.
 * round_bf16 = 1 rounds the weights and the three hidden activations to
 * BF16 (round to nearest even), as the CUDA kernels store them; sums are
 * FP64 here and FP32 on the GPU. */
static const int LP_CIN[4] = {3, 16, 16, 16}, LP_COUT[4] = {16, 16, 16, 1};
static const int LP_OFF[5] = {0, 27 * 3 * 16, 27 * 3 * 16 + 27 * 256, 27 * 3 * 16 + 2 * 27 * 256,
                              27 * 3 * 16 + 2 * 27 * 256 + 27 * 16};

static float bf16_round(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7F800000u) == 0x7F800000u) return x; /* inf / nan unchanged */
    u += 0x7FFFu + ((u >> 16) & 1u);
    u &= 0xFFFF0000u;
    float y;
    memcpy(&y, &u, 4);
    return y;
}

typedef struct {
    int nx, ny, nz;
    int64_t nc;
} lp_dims;

static inline int64_t lp_at(const lp_dims* D, int i, int j, int k) {
    if (i < 0 || j < 0 || k < 0 || i >= D->nx || j >= D->ny || k >= D->nz) return -1;
    return i + (int64_t)D->nx * (j + (int64_t)D->ny * k);
}

/* 7-point operator on the fluid cells, as the PCG uses it (walls solid) */
static void lp_apply_A(const lp_dims* D, const uint8_t* type, const double* x, double* y) {
    static const int off[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
#pragma omp parallel for schedule(static)
    for (int k = 0; k < D->nz; ++k)
        for (int j = 0; j < D->ny; ++j)
            for (int i = 0; i < D->nx; ++i) {
                int64_t id = lp_at(D, i, j, k);
                if (type[id] != NAT_FLUID) { y[id] = 0.0; continue; }
                double d = 0.0, s = 0.0;
                for (int q = 0; q < 6; ++q) {
                    int64_t n = lp_at(D, i + off[q][0], j + off[q][1], k + off[q][2]);
                    if (n < 0 || type[n] == NAT_SOLID) continue;
                    d += 1.0;
                    if (type[n] == NAT_FLUID) s += x[n];
                }
                y[id] = d * x[id] - s;
            }
}

/* one convolution layer: out[v][co] = sum_tap sum_ci W[tap][ci][co] in[v+dil*off][ci] */
static void lp_conv(const lp_dims* D, const float* in, int cin, const float* W, int cout, int dil, double* out) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < D->nz; ++k)
        for (int j = 0; j < D->ny; ++j)
            for (int i = 0; i < D->nx; ++i) {
                int64_t v = lp_at(D, i, j, k);
                double acc[16] = {0};
                for (int tap = 0; tap < 27; ++tap) {
                    int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
                    int64_t u = lp_at(D, i + dil * dx, j + dil * dy, k + dil * dz);
                    if (u < 0) continue;
                    for (int ci = 0; ci < cin; ++ci) {
                        double x = in[u * cin + ci];
                        if (x == 0.0) continue;
                        const float* w = W + (tap * cin + ci) * cout;
                        for (int co = 0; co < cout; ++co) acc[co] += (double)w[co] * x;
                    }
                }
                for (int co = 0; co < cout; ++co) out[v * cout + co] = acc[co];
            }
}

/* forward pass; keeps the inputs and activations for the backward pass */
typedef struct {
    float* in;      /* [nc][3]  */
    float* act[3];  /* [nc][16] */
    float* in0;     /* the zero-residual pass f(0): inputs and activations */
    float* act0[3];
    float* wr;      /* weights as used (rounded or not) */
    float inv_s, s;
} lp_fwd;

/* f on given input channels: hidden activations into act[], output into out[nc] (FP64 sums) */
static void lp_f(const lp_dims* D, const float* in, const float* wr, const int* dil, int round_bf16, float** act,
                 double* tmp, double* out) {
    const int64_t nc = D->nc;
    const float* cur = in;
    for (int l = 0; l < 3; ++l) {
        lp_conv(D, cur, LP_CIN[l], wr + LP_OFF[l], 16, dil[l], tmp);
        act[l] = (float*)malloc(sizeof(float) * 16 * nc);
        for (int64_t q = 0; q < 16 * nc; ++q) {
            float a = (float)(tmp[q] > 0.0 ? tmp[q] : 0.0);
            act[l][q] = round_bf16 ? bf16_round(a) : a;
        }
        cur = act[l];
    }
    lp_conv(D, cur, 16, wr + LP_OFF[3], 1, dil[3], out);
}

static void lp_forward_keep(const lp_dims* D, const uint8_t* type, const float* r, const float* w, const int* dil,
                            int round_bf16, float* z, lp_fwd* F) {
    const int64_t nc = D->nc;
    F->wr = (float*)malloc(sizeof(float) * LP_OFF[4]);
    for (int i = 0; i < LP_OFF[4]; ++i) F->wr[i] = round_bf16 ? bf16_round(w[i]) : w[i];
    double rr = 0.0, nf = 0.0;
    for (int64_t v = 0; v < nc; ++v)
        if (type[v] == NAT_FLUID) { rr += (double)r[v] * (double)r[v]; nf += 1.0; }
    F->inv_s = rr > 0.0 ? (float)(1.0 / sqrt(rr / (nf > 1.0 ? nf : 1.0))) : 1.0f;
    F->s = 1.0f / F->inv_s;
    F->in = (float*)malloc(sizeof(float) * 3 * nc);
    for (int64_t v = 0; v < nc; ++v) {
        int fl = type[v] == NAT_FLUID;
        F->in[3 * v] = fl ? r[v] * F->inv_s : 0.0f;
        F->in[3 * v + 1] = fl ? 1.0f : 0.0f;
        F->in[3 * v + 2] = type[v] == NAT_SOLID ? 1.0f : 0.0f;
    }
    F->in0 = (float*)malloc(sizeof(float) * 3 * nc);
    for (int64_t v = 0; v < nc; ++v) {
        F->in0[3 * v] = 0.0f;
        F->in0[3 * v + 1] = F->in[3 * v + 1];
        F->in0[3 * v + 2] = F->in[3 * v + 2];
    }
    double* tmp = (double*)malloc(sizeof(double) * 16 * nc);
    double* o = (double*)malloc(sizeof(double) * nc);
    double* o0 = (double*)malloc(sizeof(double) * nc);
    lp_f(D, F->in, F->wr, dil, round_bf16, F->act, tmp, o);
    lp_f(D, F->in0, F->wr, dil, round_bf16, F->act0, tmp, o0);
    /* the GPU rounds f(0) to FP32 before the subtraction */
    for (int64_t v = 0; v < nc; ++v)
        z[v] = type[v] == NAT_FLUID ? (float)((double)(float)o[v] - (double)(float)o0[v]) * F->s : 0.0f;
    free(tmp);
    free(o);
    free(o0);
}

static void lp_fwd_free(lp_fwd* F) {
    free(F->in);
    free(F->in0);
    for (int l = 0; l < 3; ++l) {
        free(F->act[l]);
        free(F->act0[l]);
    }
    free(F->wr);
}

int orc_lp_num_weights(void) { return LP_OFF[4]; }

void orc_lp_forward(int nx, int ny, int nz, const uint8_t* type, const float* r, const float* w, const int* dil,
                    int round_bf16, float* z, double* inv_s) {
    lp_dims D = {nx, ny, nz, (int64_t)nx * ny * nz};
    lp_fwd F;
    lp_forward_keep(&D, type, r, w, dil, round_bf16, z, &F);
    if (inv_s) *inv_s = F.inv_s;
    lp_fwd_free(&F);
}

/* dW[tap][ci][co] += sum_v g[v][co] in[v+dil*off][ci] */
static void lp_wgrad(const lp_dims* D, const double* g, int cout, const float* in, int cin, int dil, double* dw) {
    const int nw = 27 * cin * cout;
#pragma omp parallel
    {
        double* loc = (double*)calloc((size_t)nw, sizeof(double));
#pragma omp for schedule(static)
        for (int k = 0; k < D->nz; ++k)
            for (int j = 0; j < D->ny; ++j)
                for (int i = 0; i < D->nx; ++i) {
                    int64_t v = lp_at(D, i, j, k);
                    for (int tap = 0; tap < 27; ++tap) {
                        int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
                        int64_t u = lp_at(D, i + dil * dx, j + dil * dy, k + dil * dz);
                        if (u < 0) continue;
                        for (int co = 0; co < cout; ++co) {
                            double gv = g[v * cout + co];
                            if (gv == 0.0) continue;
                            for (int ci = 0; ci < cin; ++ci) loc[(tap * cin + ci) * cout + co] += gv * in[u * cin + ci];
                        }
                    }
                }
#pragma omp critical
        for (int q = 0; q < nw; ++q) dw[q] += loc[q];
        free(loc);
    }
}

/* gin[u][ci] = mask(u,ci) * sum_tap sum_co W[tap][ci][co] g[u - dil*off][co] */
static void lp_dgrad(const lp_dims* D, const double* g, int cout, const float* W, int cin, int dil, const float* act,
                     double* gin) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < D->nz; ++k)
        for (int j = 0; j < D->ny; ++j)
            for (int i = 0; i < D->nx; ++i) {
                int64_t u = lp_at(D, i, j, k);
                double acc[16] = {0};
                for (int tap = 0; tap < 27; ++tap) {
                    int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
                    int64_t v = lp_at(D, i - dil * dx, j - dil * dy, k - dil * dz);
                    if (v < 0) continue;
                    for (int co = 0; co < cout; ++co) {
                        double gv = g[v * cout + co];
                        if (gv == 0.0) continue;
                        for (int ci = 0; ci < cin; ++ci) acc[ci] += (double)W[(tap * cin + ci) * cout + co] * gv;
                    }
                }
                for (int ci = 0; ci < cin; ++ci) gin[u * cin + ci] = act[u * cin + ci] > 0.0f ? acc[ci] : 0.0;
            }
}

/* Jacobi diagonal inverse 1/d on fluid cells (d = non-solid neighbours, walls solid), 0 elsewhere */
static void lp_dinv(const lp_dims* D, const uint8_t* type, double* dinv) {
    static const int off[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    for (int k = 0; k < D->nz; ++k)
        for (int j = 0; j < D->ny; ++j)
            for (int i = 0; i < D->nx; ++i) {
                int64_t id = lp_at(D, i, j, k);
                double d = 0.0;
                if (type[id] == NAT_FLUID)
                    for (int q = 0; q < 6; ++q) {
                        int64_t n = lp_at(D, i + off[q][0], j + off[q][1], k + off[q][2]);
                        if (n >= 0 && type[n] != NAT_SOLID) d += 1.0;
                    }
                dinv[id] = d > 0.0 ? 1.0 / d : 0.0;
            }
}

/* Training loss of the learned preconditioner M(r) = N(r) + D^-1 r for a
 * sample (r, e) with A e = r (e = x* - x_k from a solver run, or white
 * noise): the A-norm error of M(r) as an approximation of e, relative to
 * e's own,
 *     L = |M(r) - e|_A^2 / |e|_A^2 = (m.Am - 2 m.r) / e.r + 1,
 * evaluated with the given r and e (e.r normalises).  Returns L; z = N(r)
 * (the network output alone) and the gradient with respect to the
 * (unrounded) weights out; the BF16 roundings pass the gradient straight
 * through.  dL/dN = 2 (A m - r) / e.r on the fluid cells. */
double orc_lp_loss_grad(int nx, int ny, int nz, const uint8_t* type, const float* r, const float* ev, const float* w,
                        const int* dil, int round_bf16, float* z, double* grad) {
    lp_dims D = {nx, ny, nz, (int64_t)nx * ny * nz};
    const int64_t nc = D.nc;
    lp_fwd F;
    lp_forward_keep(&D, type, r, w, dil, round_bf16, z, &F);
    double* m = (double*)malloc(sizeof(double) * nc);
    double* am = (double*)malloc(sizeof(double) * nc);
    double* dinv = (double*)malloc(sizeof(double) * nc);
    double* gz = (double*)malloc(sizeof(double) * nc);
    lp_dinv(&D, type, dinv);
    for (int64_t v = 0; v < nc; ++v) m[v] = type[v] == NAT_FLUID ? (double)z[v] + dinv[v] * (double)r[v] : 0.0;
    lp_apply_A(&D, type, m, am);
    double mam = 0.0, mr = 0.0, er = 0.0;
    for (int64_t v = 0; v < nc; ++v) {
        if (type[v] != NAT_FLUID) continue;
        mam += m[v] * am[v];
        mr += m[v] * (double)r[v];
        er += (double)ev[v] * (double)r[v];
    }
    const double loss = (mam - 2.0 * mr) / er + 1.0;
    if (grad) {
        memset(grad, 0, sizeof(double) * LP_OFF[4]);
        /* dL/d(out of layer 3) = s dL/dN */
        for (int64_t v = 0; v < nc; ++v)
            gz[v] = type[v] == NAT_FLUID ? 2.0 * (am[v] - (double)r[v]) / er * (double)F.s : 0.0;
        double* g = (double*)malloc(sizeof(double) * 16 * nc);
        double* g2 = (double*)malloc(sizeof(double) * 16 * nc);
        /* through f(r/s) with +gz, then through f(0) with -gz */
        for (int path = 0; path < 2; ++path) {
            float** act = path ? F.act0 : F.act;
            const float* in = path ? F.in0 : F.in;
            if (path)
                for (int64_t v = 0; v < nc; ++v) gz[v] = -gz[v];
            lp_wgrad(&D, gz, 1, act[2], 16, dil[3], grad + LP_OFF[3]);
            lp_dgrad(&D, gz, 1, F.wr + LP_OFF[3], 16, dil[3], act[2], g);
            lp_wgrad(&D, g, 16, act[1], 16, dil[2], grad + LP_OFF[2]);
            lp_dgrad(&D, g, 16, F.wr + LP_OFF[2], 16, dil[2], act[1], g2);
            lp_wgrad(&D, g2, 16, act[0], 16, dil[1], grad + LP_OFF[1]);
            lp_dgrad(&D, g2, 16, F.wr + LP_OFF[1], 16, dil[1], act[0], g);
            lp_wgrad(&D, g, 16, in, 3, dil[0], grad + LP_OFF[0]);
        }
        free(g);
        free(g2);
    }
    free(m);
    free(am);
    free(dinv);
    free(gz);
    lp_fwd_free(&F);
    return loss;
}

/* flexible CG (FCG(1)) with M(r) = N(r) + D^-1 r as preconditioner, in
 * FP64 apart from the network; returns iterations (max_iter + 1 if not
 * converged or stalled: less than 10% residual reduction over 16
 * iterations), x out, *rel_res = |b - A x| / |b| */
int orc_lp_fpcg(int nx, int ny, int nz, const uint8_t* type, const double* b, const float* w, const int* dil,
                int round_bf16, double tol, int max_iter, double* x, double* rel_res) {
    lp_dims D = {nx, ny, nz, (int64_t)nx * ny * nz};
    const int64_t nc = D.nc;
    double *r = (double*)calloc((size_t)nc, 8), *p = (double*)calloc((size_t)nc, 8), *q = (double*)calloc((size_t)nc, 8),
           *zd = (double*)calloc((size_t)nc, 8);
    float *rf = (float*)calloc((size_t)nc, 4), *zf = (float*)calloc((size_t)nc, 4);
    double* dinv = (double*)malloc(sizeof(double) * nc);
    lp_dinv(&D, type, dinv);
    double bb = 0.0;
    for (int64_t v = 0; v < nc; ++v) {
        x[v] = 0.0;
        r[v] = type[v] == NAT_FLUID ? b[v] : 0.0;
        bb += r[v] * r[v];
    }
    const double bn = sqrt(bb);
    int it = 0;
    double pq_prev = 0.0, rr_check = bb;
    if (bn > 0.0) {
        for (it = 1; it <= max_iter + 1; ++it) {
            for (int64_t v = 0; v < nc; ++v) rf[v] = (float)r[v];
            orc_lp_forward(nx, ny, nz, type, rf, w, dil, round_bf16, zf, NULL);
            double rzn = 0.0, zq = 0.0;
            for (int64_t v = 0; v < nc; ++v) {
                zd[v] = (double)zf[v] + dinv[v] * r[v]; /* M(r) = N(r) + D^-1 r */
                rzn += r[v] * zd[v];
                zq += zd[v] * q[v];
            }
            if (rzn == 0.0 || !isfinite(rzn)) break;
            /* FCG(1): p = z + beta p A-orthogonal to the previous p, beta = -z.q / p.q */
            const double beta = it == 1 ? 0.0 : -zq / pq_prev;
            for (int64_t v = 0; v < nc; ++v) p[v] = zd[v] + beta * p[v];
            lp_apply_A(&D, type, p, q);
            double pq = 0.0;
            for (int64_t v = 0; v < nc; ++v) pq += p[v] * q[v];
            if (!(pq > 0.0)) break;
            const double alpha = rzn / pq; /* exact line search: r is orthogonal to the previous p */
            pq_prev = pq;
            double rr = 0.0;
            for (int64_t v = 0; v < nc; ++v) {
                x[v] += alpha * p[v];
                r[v] -= alpha * q[v];
                rr += r[v] * r[v];
            }
            if (sqrt(rr) <= tol * bn) break;
            /* the GPU solve's stagnation rule: every 16 iterations the residual
             * norm must have fallen by 10% since the previous check */
            if (it % 16 == 0) {
                if (rr > 0.81 * rr_check) { it = max_iter + 1; break; }
                rr_check = rr;
            }
        }
    }
    lp_apply_A(&D, type, x, q);
    double rr = 0.0;
    for (int64_t v = 0; v < nc; ++v)
        if (type[v] == NAT_FLUID) { double d = b[v] - q[v]; rr += d * d; }
    if (rel_res) *rel_res = bn > 0.0 ? sqrt(rr) / bn : 0.0;
    free(r); free(p); free(q); free(zd); free(rf); free(zf); free(dinv);
    return it;
}

/* ============================== multilevel preconditioner (method 2) ====
 * One V-cycle over 2x coarsened grids with the network as the coarsest
 * solve (no reference counterpart; the GPU form is flip2_b200/csrc/mg.cu).
 * Level l+1 has ceil(n_l / 2) cells per axis, padded to a multiple of 8 with
 * solid cells, until every axis has at most 16.  A coarse cell is air if any
 * child is air, else fluid if any child is fluid, else solid.  Damped Jacobi
 * (omega = 2/3): two sweeps from zero before the restriction (1/2 x the sum
 * of the 8 children's residuals), two after adding the parent's correction;
 * the coarsest level starts from N(r) + D^-1 r (network) or omega D^-1 r
 * (mode 1) and takes two sweeps.  FP64 apart from the network. */
#define MG_MAX_LEVELS 8
#define MG_COARSEST 16
#define MG_OMEGA (2.0 / 3.0)

typedef struct {
    lp_dims D; /* padded */
    int ex, ey, ez;
    uint8_t* type;
    double *dinv, *r, *z, *t;
} mg_level;

static int mg_levels_plan(int nx, int ny, int nz, mg_level* L) {
    int ex = nx, ey = ny, ez = nz, n = 0;
    while (n < MG_MAX_LEVELS) {
        mg_level* l = &L[n];
        memset(l, 0, sizeof(*l));
        l->ex = ex; l->ey = ey; l->ez = ez;
        l->D.nx = (ex + 7) & ~7; l->D.ny = (ey + 7) & ~7; l->D.nz = (ez + 7) & ~7;
        l->D.nc = (int64_t)l->D.nx * l->D.ny * l->D.nz;
        ++n;
        if (ex <= MG_COARSEST && ey <= MG_COARSEST && ez <= MG_COARSEST) break;
        ex = (ex + 1) / 2; ey = (ey + 1) / 2; ez = (ez + 1) / 2;
    }
    return n;
}

static void mg_coarsen(const mg_level* F, mg_level* C) {
    for (int K = 0; K < C->D.nz; ++K)
        for (int J = 0; J < C->D.ny; ++J)
            for (int I = 0; I < C->D.nx; ++I) {
                uint8_t t = NAT_SOLID;
                if (I < C->ex && J < C->ey && K < C->ez) {
                    int air = 0, fluid = 0;
                    for (int c = 0; c < 8; ++c) {
                        int i = 2 * I + (c & 1), j = 2 * J + ((c >> 1) & 1), k = 2 * K + (c >> 2);
                        if (i >= F->ex || j >= F->ey || k >= F->ez) continue;
                        uint8_t ft = F->type[lp_at(&F->D, i, j, k)];
                        air |= ft == NAT_AIR;
                        fluid |= ft == NAT_FLUID;
                    }
                    t = air ? NAT_AIR : (fluid ? NAT_FLUID : NAT_SOLID);
                }
                C->type[lp_at(&C->D, I, J, K)] = t;
            }
}

/* out = in + omega D^-1 (r - A in) on the fluid cells of L */
static void mg_sweep(const mg_level* L, const double* in, double* out, double* tmp) {
    lp_apply_A(&L->D, L->type, in, tmp);
    for (int64_t v = 0; v < L->D.nc; ++v)
        out[v] = L->type[v] == NAT_FLUID ? in[v] + MG_OMEGA * L->dinv[v] * (L->r[v] - tmp[v]) : 0.0;
}

static void mg_vcycle(mg_level* L, int levels, int l, const float* w, const int* dil, int round_bf16, int mode) {
    mg_level* f = &L[l];
    const int64_t nc = f->D.nc;
    double* tmp = (double*)malloc(sizeof(double) * nc);
    double* t2 = (double*)malloc(sizeof(double) * nc);
    if (l == levels - 1) {
        if (mode == 0) {
            float* rf = (float*)malloc(sizeof(float) * nc);
            float* zf = (float*)malloc(sizeof(float) * nc);
            for (int64_t v = 0; v < nc; ++v) rf[v] = (float)f->r[v];
            orc_lp_forward(f->D.nx, f->D.ny, f->D.nz, f->type, rf, w, dil, round_bf16, zf, NULL);
            for (int64_t v = 0; v < nc; ++v) t2[v] = f->type[v] == NAT_FLUID ? (double)zf[v] + f->dinv[v] * f->r[v] : 0.0;
            free(rf);
            free(zf);
        } else {
            for (int64_t v = 0; v < nc; ++v) t2[v] = f->type[v] == NAT_FLUID ? MG_OMEGA * f->dinv[v] * f->r[v] : 0.0;
        }
        mg_sweep(f, t2, f->t, tmp);
        mg_sweep(f, f->t, f->z, tmp);
    } else {
        mg_level* c = &L[l + 1];
        for (int64_t v = 0; v < nc; ++v) t2[v] = f->type[v] == NAT_FLUID ? MG_OMEGA * f->dinv[v] * f->r[v] : 0.0;
        mg_sweep(f, t2, f->t, tmp);
        lp_apply_A(&f->D, f->type, f->t, tmp);
        for (int64_t v = 0; v < c->D.nc; ++v) c->r[v] = 0.0;
        for (int k = 0; k < f->D.nz; ++k)
            for (int j = 0; j < f->D.ny; ++j)
                for (int i = 0; i < f->D.nx; ++i) {
                    int64_t v = lp_at(&f->D, i, j, k);
                    if (f->type[v] != NAT_FLUID) continue;
                    int64_t p = lp_at(&c->D, i >> 1, j >> 1, k >> 1);
                    if (c->type[p] == NAT_FLUID) c->r[p] += 0.5 * (f->r[v] - tmp[v]);
                }
        mg_vcycle(L, levels, l + 1, w, dil, round_bf16, mode);
        for (int k = 0; k < f->D.nz; ++k)
            for (int j = 0; j < f->D.ny; ++j)
                for (int i = 0; i < f->D.nx; ++i) {
                    int64_t v = lp_at(&f->D, i, j, k);
                    t2[v] = f->type[v] == NAT_FLUID ? f->t[v] + c->z[lp_at(&c->D, i >> 1, j >> 1, k >> 1)] : 0.0;
                }
        mg_sweep(f, t2, f->t, tmp);
        mg_sweep(f, f->t, f->z, tmp);
    }
    free(tmp);
    free(t2);
}

typedef struct {
    int levels;
    mg_level L[MG_MAX_LEVELS];
} mg_hier;

static void mg_hier_init(mg_hier* H, int nx, int ny, int nz, const uint8_t* type) {
    H->levels = mg_levels_plan(nx, ny, nz, H->L);
    for (int l = 0; l < H->levels; ++l) {
        mg_level* c = &H->L[l];
        const int64_t nc = c->D.nc;
        c->type = (uint8_t*)malloc(nc);
        c->dinv = (double*)malloc(sizeof(double) * nc);
        c->r = (double*)calloc((size_t)nc, 8);
        c->z = (double*)calloc((size_t)nc, 8);
        c->t = (double*)calloc((size_t)nc, 8);
        if (l == 0) memcpy(c->type, type, (size_t)nc);
        else mg_coarsen(&H->L[l - 1], c);
        lp_dinv(&c->D, c->type, c->dinv);
    }
}
static void mg_hier_free(mg_hier* H) {
    for (int l = 0; l < H->levels; ++l) {
        mg_level* c = &H->L[l];
        free(c->type); free(c->dinv); free(c->r); free(c->z); free(c->t);
    }
}

int orc_mg_levels(int nx, int ny, int nz, int* dims) {
    mg_level L[MG_MAX_LEVELS];
    int n = mg_levels_plan(nx, ny, nz, L);
    for (int l = 0; l < n && dims; ++l) {
        dims[3 * l] = L[l].D.nx; dims[3 * l + 1] = L[l].D.ny; dims[3 * l + 2] = L[l].D.nz;
    }
    return n;
}

void orc_mg_apply(int nx, int ny, int nz, const uint8_t* type, const float* r, const float* w, const int* dil,
                  int round_bf16, int mode, double* z) {
    mg_hier H;
    mg_hier_init(&H, nx, ny, nz, type);
    const int64_t nc = H.L[0].D.nc;
    for (int64_t v = 0; v < nc; ++v) H.L[0].r[v] = type[v] == NAT_FLUID ? (double)r[v] : 0.0;
    mg_vcycle(H.L, H.levels, 0, w, dil, round_bf16, mode);
    memcpy(z, H.L[0].z, sizeof(double) * nc);
    mg_hier_free(&H);
}

/* FCG(1) with the V-cycle as preconditioner; the same loop and stagnation
 * rule as orc_lp_fpcg */
int orc_mg_fcg(int nx, int ny, int nz, const uint8_t* type, const double* b, const float* w, const int* dil,
               int round_bf16, int mode, double tol, int max_iter, double* x, double* rel_res) {
    lp_dims D = {nx, ny, nz, (int64_t)nx * ny * nz};
    const int64_t nc = D.nc;
    mg_hier H;
    mg_hier_init(&H, nx, ny, nz, type);
    double *r = (double*)calloc((size_t)nc, 8), *p = (double*)calloc((size_t)nc, 8), *q = (double*)calloc((size_t)nc, 8);
    double bb = 0.0;
    for (int64_t v = 0; v < nc; ++v) {
        x[v] = 0.0;
        r[v] = type[v] == NAT_FLUID ? b[v] : 0.0;
        bb += r[v] * r[v];
    }
    const double bn = sqrt(bb);
    int it = 0;
    double pq_prev = 0.0, rr_check = bb;
    if (bn > 0.0) {
        for (it = 1; it <= max_iter + 1; ++it) {
            /* the GPU's V-cycle reads r in FP32 */
            for (int64_t v = 0; v < nc; ++v) H.L[0].r[v] = (double)(float)r[v];
            mg_vcycle(H.L, H.levels, 0, w, dil, round_bf16, mode);
            const double* zd = H.L[0].z;
            double rzn = 0.0, zq = 0.0;
            for (int64_t v = 0; v < nc; ++v) {
                rzn += r[v] * zd[v];
                zq += zd[v] * q[v];
            }
            if (rzn == 0.0 || !isfinite(rzn)) break;
            const double beta = it == 1 ? 0.0 : -zq / pq_prev;
            for (int64_t v = 0; v < nc; ++v) p[v] = zd[v] + beta * p[v];
            lp_apply_A(&D, type, p, q);
            double pq = 0.0;
            for (int64_t v = 0; v < nc; ++v) pq += p[v] * q[v];
            if (!(pq > 0.0)) break;
            const double alpha = rzn / pq;
            pq_prev = pq;
            double rr = 0.0;
            for (int64_t v = 0; v < nc; ++v) {
                x[v] += alpha * p[v];
                r[v] -= alpha * q[v];
                rr += r[v] * r[v];
            }
            if (sqrt(rr) <= tol * bn) break;
            if (it % 16 == 0) {
                if (rr > 0.81 * rr_check) { it = max_iter + 1; break; }
                rr_check = rr;
            }
        }
    }
    lp_apply_A(&D, type, x, q);
    double rr = 0.0;
    for (int64_t v = 0; v < nc; ++v)
        if (type[v] == NAT_FLUID) { double d = b[v] - q[v]; rr += d * d; }
    if (rel_res) *rel_res = bn > 0.0 ? sqrt(rr) / bn : 0.0;
    free(r); free(p); free(q);
    mg_hier_free(&H);
    return it;
}
