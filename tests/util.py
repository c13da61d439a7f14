"""Helpers shared by the tests (host-side conversions and comparisons)."""
import numpy as np


def tiled_to_linear(a, nx, ny, nz):
    """Tile-blocked slot array (slot = tile*512 + (i&7) + 8(j&7) + 64(k&7)) ->
    x-fastest linear array of nx*ny*nz."""
    tx, ty = nx // 8, ny // 8
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    tile = (i >> 3) + tx * ((j >> 3) + ty * (k >> 3))
    slot = tile * 512 + (i & 7) + 8 * (j & 7) + 64 * (k & 7)
    return np.asarray(a)[slot.ravel()]


def rel_err(a, b, floor=0.0):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = max(np.max(np.abs(b)), floor)
    if den == 0.0:
        return float(np.max(np.abs(a)))
    return float(np.max(np.abs(a - b)) / den)


def sealed_pockets(typ, shape):
    """Labels of the fluid regions that touch no air cell (x fastest; 0 air,
    1 fluid, 2 solid, outside the box solid) and their count.  The pressure
    of such a region has pure Neumann boundaries: it is defined only up to a
    constant, and different solvers that all meet the residual tolerance may
    leave different constants there."""
    from scipy import ndimage
    nx, ny, nz = shape
    t = np.asarray(typ).reshape(nz, ny, nx)
    lab, n = ndimage.label(t == 1)
    air = t == 0
    near_air = np.zeros_like(air)
    for ax in range(3):
        near_air |= np.roll(air, 1, ax) & (np.arange(t.shape[ax]).reshape([-1 if a == ax else 1 for a in range(3)]) > 0)
        near_air |= np.roll(air, -1, ax) & (np.arange(t.shape[ax]).reshape([-1 if a == ax else 1 for a in range(3)])
                                            < t.shape[ax] - 1)
    anchored = np.unique(lab[near_air & (lab > 0)])
    sealed = np.setdiff1d(np.arange(1, n + 1), anchored)
    pocket = np.where(np.isin(lab, sealed), lab, 0)
    return pocket.ravel(), int(sealed.size)


def remove_pocket_constants(x, ref, pocket):
    """x with each sealed pocket shifted by the mean of ref - x over it."""
    x = np.asarray(x, np.float64).copy()
    for p in np.unique(pocket[pocket > 0]):
        m = pocket == p
        x[m] += float(np.mean(np.asarray(ref, np.float64)[m] - x[m]))
    return x


def u32(t):
    """torch int32 tensor holding u32 bits -> numpy uint32."""
    return t.cpu().numpy().view(np.uint32)


def zapron_race_voxels(b, g):
    """Voxels whose reference divergence is not deterministic.

    The reference's z-apron copy writes target (tz, y, tz) -- x replaced by z
    (voxelSolveFunctions.cu:85) -- so up to eight source voxels of one row land
    on one shared-memory word through plain `+=` from different threads
    (voxelSolveFunctions.cu:48-93): the surviving sum depends on the warp
    schedule.  Returns a bool mask over the compacted voxels whose divergence
    reads such a word."""
    nv, ids, keys, st, yt = b["node_voxels"], b["voxel_ids"], b["sorted_keys"], b["starts"], b["ytable"]
    nodes = int(b["nodes"])
    X, Y = g.sizeX, g.sizeY
    aff = np.zeros(int(b["voxels"]), bool)
    for nd in range(nodes):
        vs = int(nv[nd - 1]) if nd else 0
        ve = int(nv[nd])
        cur = int(keys[st[nd]])
        cy, cz = (cur % (X * Y)) // X, cur // (X * Y)
        if cz < 1 or yt[(cz - 1) * Y + cy] >= nodes:
            continue
        nid = int(yt[(cz - 1) * Y + cy])
        s0 = int(nv[nid - 1]) if nid else 0
        src = ids[s0:int(nv[nid])].astype(np.int64)
        sy, sz = (src % 64) // 8, src // 64
        t = (sz - 4) + sy * 8 + (sz - 4) * 64
        t = t[sz >= 4]
        u, c = np.unique(t, return_counts=True)
        T = set(u[c >= 2].tolist())
        if not T:
            continue
        v = ids[vs:ve].astype(np.int64)
        aff[vs:ve] = [(a in T) or (a + 1 in T) or (a + 8 in T) or (a + 64 in T) for a in v]
    return aff


def native_step_errors(P, ref, nc, F):
    """Errors of a native step run on the engine P against the FP64 oracle
    run `ref` (oracle.nat_step of the same input) on an nc^3 grid of cell
    1/nc.  Every quantity is measured in the norm the parity tests bound:
      pressure_rel_err_max   max |phi - phi64| / max |phi64| (fluid cells);
      p2g_face_rel_err       max over u, v, w of |U - U64|, divided by the
                             largest |U64| over all three (the face grids
                             right after P2G: one scale for the vector
                             field, so that a component that is zero up to
                             rounding, like w of a dam break spanning the box
                             in z, is not measured against its own noise);
      proj_face_rel_err      the same for the faces after the projection, the
                             grid velocity that G2P samples;
      velocity_rel_err_max   max |v - v64| / max |v64| over the particles;
      position_err_max_in_h  max |x - x64| / h."""
    import numpy as np
    perm = P.read(F.BUF_PERM)
    phi = tiled_to_linear(P.read(F.BUF_PRESSURE), nc, nc, nc).astype(np.float64)
    out = {}
    fl = np.abs(ref["phi"]) > 0
    out["pressure_rel_err_max"] = rel_err(phi, ref["phi"])
    out["pressure_rel_err_l2"] = float(np.linalg.norm(phi[fl] - ref["phi"][fl]) / max(np.linalg.norm(ref["phi"][fl]), 1e-300))
    dp2g = dproj = 0.0
    sp2g = sproj = 0.0
    for (bp, bq, kp, kq) in ((F.BUF_GRID_U_P2G, F.BUF_GRID_U, "u", "u_proj"), (F.BUF_GRID_V_P2G, F.BUF_GRID_V, "v", "v_proj"),
                             (F.BUF_GRID_W_P2G, F.BUF_GRID_W, "w", "w_proj")):
        g = tiled_to_linear(P.read(bp, np.float32), nc, nc, nc).astype(np.float64)
        dp2g, sp2g = max(dp2g, float(np.max(np.abs(g - ref[kp])))), max(sp2g, float(np.max(np.abs(ref[kp]))))
        g = tiled_to_linear(P.read(bq, np.float32), nc, nc, nc).astype(np.float64)
        dproj, sproj = max(dproj, float(np.max(np.abs(g - ref[kq])))), max(sproj, float(np.max(np.abs(ref[kq]))))
    out["p2g_face_rel_err"] = dp2g / sp2g if sp2g > 0 else dp2g
    out["proj_face_rel_err"] = dproj / sproj if sproj > 0 else dproj
    pg, vg = P.download()
    po, vo = ref["pos"][perm], ref["vel"][perm]
    out["velocity_rel_err_max"] = rel_err(vg, vo)
    out["position_err_max_in_h"] = float(np.max(np.abs(pg.astype(np.float64) - po)) * nc)
    return out
