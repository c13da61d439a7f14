"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by the smoke check in
__graft_entry__.py and by bench.py's CPU-baseline leg; never by the product
package.  See flip_oracle.h for what each function restates.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
i8p = np.ctypeslib.ndpointer(np.int8, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class Grid(C.Structure):
    """Mirror of class Grid (engine/grid.hpp:8-38)."""
    _fields_ = [("negX", C.c_float), ("negY", C.c_float), ("negZ", C.c_float),
                ("sizeX", C.c_uint32), ("sizeY", C.c_uint32), ("sizeZ", C.c_uint32),
                ("cellSize", C.c_float)]


class RefStepInfo(C.Structure):
    _fields_ = [("nodes", C.c_uint32), ("voxels", C.c_uint32), ("gs_iters_total", C.c_uint32),
                ("dt", C.c_double), ("residual", C.c_double)]


class NatParams(C.Structure):
    _fields_ = [("ox", C.c_double), ("oy", C.c_double), ("oz", C.c_double), ("h", C.c_double),
                ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("gravity_y", C.c_double), ("flip", C.c_double), ("dt", C.c_double), ("tol", C.c_double),
                ("max_iter", C.c_int32), ("solid_u", C.c_double), ("solid_v", C.c_double), ("solid_w", C.c_double)]


class NatInfo(C.Structure):
    _fields_ = [("iters", C.c_int32), ("rel_residual", C.c_double), ("fluid_cells", C.c_int64)]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so is not built (make -C oracle)")
        L = C.CDLL(path)
        I64, U32, D, I = C.c_int64, C.c_uint32, C.c_double, C.c_int
        sig = {
            "orc_ref_keys": (None, [I64, f64p, f64p, f64p, Grid, u32p]),
            "orc_ref_grid_cell_checks": (I64, [u32p, u32p, C.c_uint64, C.POINTER(C.c_uint64)]),
            "orc_sort_pairs": (None, [I64, u32p, u32p, u32p]),
            "orc_sort_pairs_payload": (None, [I64, u32p, u32p, u32p, u32p]),
            "orc_inclusive_scan": (None, [I64, u32p]),
            "orc_gather_f64": (None, [I64, u32p, f64p, f64p]),
            "orc_mark_unique_scan": (U32, [I64, u32p, u32p]),
            "orc_cell_starts": (None, [I64, u32p, u32p]),
            "orc_ydim_rows": (None, [U32, u32p, u32p, Grid, u32p]),
            "orc_ref_voxel_counts": (None, [U32, I64, u32p, u32p, f64p, f64p, f64p, Grid, u32p]),
            "orc_ref_voxel_ids": (None, [U32, I64, u32p, u32p, f64p, f64p, f64p, Grid, u32p, u32p, i8p]),
            "orc_ref_p2g": (None, [U32, I64, u32p, u32p, f64p, f64p, f64p, f64p, u32p, u32p, i8p, Grid, I, f64p]),
            "orc_ref_g2p": (None, [U32, I64, u32p, u32p, f64p, f64p, f64p, u32p, u32p, f64p, Grid, I, f64p]),
            "orc_ref_advect": (None, [I64, D, f64p, f64p]),
            "orc_ref_move_solids_targets": (None, [U32, I64, u32p, u32p, f64p, f64p, f64p, u32p, u32p, i8p, Grid, u32p]),
            "orc_ref_getmax": (D, [I64, f64p, I]),
            "orc_ref_gravity": (None, [I64, i8p, f64p, D, I]),
            "orc_ref_divergence": (None, [U32, u32p, u32p, f64p, f64p, f64p, Grid, u32p, u32p, u32p, f64p]),
            "orc_ref_gs_pass": (None, [U32, u32p, u32p, i8p, f64p, f64p, f64p, D, D, Grid, I, D]),
            "orc_ref_gs_solve": (D, [U32, u32p, u32p, i8p, f64p, f64p, f64p, D, D, Grid, D, U32, C.POINTER(U32)]),
            "orc_ref_velocity_update": (None, [U32, u32p, u32p, i8p, f64p, f64p, f64p, f64p, D, D, Grid]),
            "orc_ref_substep": (I, [I64, f64p, f64p, f64p, f64p, f64p, f64p, Grid, D, D, I, C.POINTER(RefStepInfo)]),
            "orc_nat_keys": (None, [I64, f32p, C.POINTER(NatParams), u32p]),
            "orc_nat_step": (I, [I64, f32p, f32p, C.c_void_p, C.POINTER(NatParams), f64p, f64p, f64p, f64p, C.POINTER(NatInfo)]),
            "orc_nat_step_ex": (I, [I64, f32p, f32p, C.c_void_p, C.POINTER(NatParams), f64p, f64p, f64p, f64p, f64p, f64p,
                                    f64p, C.POINTER(NatInfo)]),
            "orc_nat_p2g": (None, [I64, f32p, f32p, C.POINTER(NatParams), f64p, f64p, f64p, u8p]),
            "orc_nat_pcg": (I, [u8p, f64p, f64p, C.POINTER(NatParams), C.POINTER(D)]),
            "orc_nat_apply_A": (None, [u8p, f64p, f64p, C.POINTER(NatParams)]),
            "orc_lp_num_weights": (I, []),
            "orc_lp_forward": (None, [I, I, I, u8p, f32p, f32p, i32p, I, f32p, C.POINTER(D)]),
            "orc_lp_loss_grad": (D, [I, I, I, u8p, f32p, f32p, f32p, i32p, I, f32p, f64p]),
            "orc_lp_fpcg": (I, [I, I, I, u8p, f64p, f32p, i32p, I, D, I, f64p, C.POINTER(D)]),
            "orc_mg_levels": (I, [I, I, I, i32p]),
            "orc_mg_apply": (None, [I, I, I, u8p, f32p, f32p, i32p, I, I, f64p]),
            "orc_mg_fcg": (I, [I, I, I, u8p, f64p, f32p, i32p, I, I, D, I, f64p, C.POINTER(D)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def grid(negX, negY, negZ, X, Y, Z, cell):
    return Grid(negX, negY, negZ, X, Y, Z, cell)


# ------------------------------------------------------------- reference math
def ref_keys(px, py, pz, g):
    """rootCell: returns (keys, clamped px, py, pz)."""
    px, py, pz = (np.ascontiguousarray(a, np.float64).copy() for a in (px, py, pz))
    keys = np.empty(px.size, np.uint32)
    lib().orc_ref_keys(px.size, px, py, pz, g, keys)
    return keys, px, py, pz


def ref_grid_cell_checks(unsorted, sorted_keys):
    """The reference's CPU verification of its binning (engine/testing.h:25-53):
    storeGridCellMap on the unsorted cell keys, validateGridCellOrdering on the
    sorted ones.  Returns (status, cells): status 0 when ordered with equal
    per-cell counts, 1 + i at the first out-of-order index i, -m for m cells
    whose counts differ; cells = distinct cells stored."""
    u = np.ascontiguousarray(unsorted, np.uint32)
    s = np.ascontiguousarray(sorted_keys, np.uint32)
    cells = C.c_uint64(0)
    st = lib().orc_ref_grid_cell_checks(u, s, u.size, C.byref(cells))
    return int(st), int(cells.value)


def sort_pairs(keys, vals=None):
    keys = np.ascontiguousarray(keys, np.uint32)
    ko = np.empty_like(keys)
    vo = np.empty_like(keys)
    if vals is None:
        lib().orc_sort_pairs(keys.size, keys, ko, vo)
    else:
        lib().orc_sort_pairs_payload(keys.size, keys, np.ascontiguousarray(vals, np.uint32), ko, vo)
    return ko, vo


def ref_bin(px, py, pz, g):
    """alignParticlesToGrid + sortParticles + generateVoxels on host arrays.

    Returns a dict with every intermediate buffer under the reference's names.
    """
    L = lib()
    keys, px, py, pz = ref_keys(px, py, pz, g)
    skeys, perm = sort_pairs(keys)
    spx, spy, spz = px[perm], py[perm], pz[perm]
    n = keys.size
    flags = np.empty(n, np.uint32)
    nodes = L.orc_mark_unique_scan(n, skeys, flags)
    starts = np.empty(max(nodes, 1), np.uint32)
    L.orc_cell_starts(n, flags, starts)
    starts = starts[:nodes]
    ytab = np.empty(g.sizeY * g.sizeZ, np.uint32)
    L.orc_ydim_rows(nodes, starts, skeys, g, ytab)
    counts = np.empty(max(nodes, 1), np.uint32)
    L.orc_ref_voxel_counts(nodes, n, starts, skeys, spx, spy, spz, g, counts)
    counts = counts[:nodes]
    node_voxels = np.cumsum(counts, dtype=np.uint64).astype(np.uint32)
    nvox = int(node_voxels[-1]) if nodes else 0
    ids = np.empty(max(nvox, 1), np.uint32)
    sol = np.empty(max(nvox, 1), np.int8)
    L.orc_ref_voxel_ids(nodes, n, starts, skeys, spx, spy, spz, g, node_voxels, ids, sol)
    return dict(keys=keys, px=px, py=py, pz=pz, sorted_keys=skeys, perm=perm, spx=spx, spy=spy, spz=spz,
                flags=flags, nodes=nodes, starts=starts, ytable=ytab, counts=counts,
                node_voxels=node_voxels, voxels=nvox, voxel_ids=ids[:nvox], solids=sol[:nvox])


def ref_p2g(b, v, g, dim):
    out = np.empty(max(b["voxels"], 1), np.float64)
    lib().orc_ref_p2g(b["nodes"], b["sorted_keys"].size, b["starts"], b["sorted_keys"], b["spx"], b["spy"], b["spz"],
                      np.ascontiguousarray(v, np.float64), b["node_voxels"], b["voxel_ids"], b["solids"], g, dim, out)
    return out[:b["voxels"]]


def ref_g2p(b, px, py, pz, voxel_u, g, dim):
    out = np.empty(b["sorted_keys"].size, np.float64)
    lib().orc_ref_g2p(b["nodes"], out.size, b["starts"], b["sorted_keys"], np.ascontiguousarray(px), np.ascontiguousarray(py),
                      np.ascontiguousarray(pz), b["node_voxels"], b["voxel_ids"],
                      np.ascontiguousarray(voxel_u, np.float64), g, dim, out)
    return out


def ref_getmax(a, absolute=True):
    a = np.ascontiguousarray(a, np.float64)
    return lib().orc_ref_getmax(a.size, a, 1 if absolute else 0)


def ref_divergence(b, ux, uy, uz, g):
    out = np.empty(max(b["voxels"], 1), np.float64)
    lib().orc_ref_divergence(b["nodes"], b["node_voxels"], b["voxel_ids"], np.ascontiguousarray(ux), np.ascontiguousarray(uy),
                             np.ascontiguousarray(uz), g, b["ytable"], b["starts"], b["sorted_keys"], out)
    return out[:b["voxels"]]


def ref_gravity(b, uy, dt, remove=False):
    uy = np.ascontiguousarray(uy, np.float64).copy()
    lib().orc_ref_gravity(uy.size, b["solids"], uy, dt, 1 if remove else 0)
    return uy


def ref_gs_pass(b, divU, p, dt, red, density=0.014, w=1.9, g=None):
    p = np.ascontiguousarray(p, np.float64).copy()
    res = np.zeros_like(p)
    lib().orc_ref_gs_pass(b["nodes"], b["node_voxels"], b["voxel_ids"], b["solids"], np.ascontiguousarray(divU),
                          p, res, density, dt, g, 1 if red else 0, w)
    return p, res


def ref_gs_solve(b, divU, p, dt, g, density=0.014, threshold=0.01, max_iter=16384):
    p = np.ascontiguousarray(p, np.float64).copy()
    res = np.zeros_like(p)
    it = C.c_uint32(0)
    r = lib().orc_ref_gs_solve(b["nodes"], b["node_voxels"], b["voxel_ids"], b["solids"], np.ascontiguousarray(divU),
                               p, res, density, dt, g, threshold, max_iter, C.byref(it))
    return r, it.value, p, res


def ref_velocity_update(b, p, ux, uy, uz, dt, g, density=0.014):
    ux, uy, uz = (np.ascontiguousarray(a, np.float64).copy() for a in (ux, uy, uz))
    lib().orc_ref_velocity_update(b["nodes"], b["node_voxels"], b["voxel_ids"], b["solids"], np.ascontiguousarray(p),
                                  ux, uy, uz, dt, density, g)
    return ux, uy, uz


def ref_move_targets(b, px, py, pz, g):
    out = np.empty(b["sorted_keys"].size, np.uint32)
    lib().orc_ref_move_solids_targets(b["nodes"], out.size, b["starts"], b["sorted_keys"], np.ascontiguousarray(px),
                                      np.ascontiguousarray(py), np.ascontiguousarray(pz), b["node_voxels"],
                                      b["voxel_ids"], b["solids"], g, out)
    return out


def ref_substep(px, py, pz, vx, vy, vz, g, frame_dt=1.0 / 24.0, elapsed=0.0, permute_velocities=False):
    arrs = [np.ascontiguousarray(a, np.float64).copy() for a in (px, py, pz, vx, vy, vz)]
    info = RefStepInfo()
    rc = lib().orc_ref_substep(arrs[0].size, *arrs, g, frame_dt, elapsed, 1 if permute_velocities else 0, C.byref(info))
    if rc != 0:
        raise RuntimeError("orc_ref_substep failed")
    return arrs, info


# ---------------------------------------------------------- native-mode step
def nat_params(nx, ny, nz, h, origin=(0.0, 0.0, 0.0), gravity_y=-9.8, flip=0.95, dt=1.0 / 240, tol=1e-6, max_iter=4000,
               solid_velocity=(0.0, 0.0, 0.0)):
    return NatParams(origin[0], origin[1], origin[2], h, nx, ny, nz, gravity_y, flip, dt, tol, max_iter, *solid_velocity)


def nat_keys(pos, P):
    pos = np.ascontiguousarray(pos, np.float32)
    keys = np.empty(pos.shape[0], np.uint32)
    lib().orc_nat_keys(pos.shape[0], pos, C.byref(P), keys)
    return keys


def nat_step(pos, vel, P, solid=None):
    """One native-mode step in FP64.  pos/vel: (n,3) float32, updated copies
    returned, with the face grids after P2G (u, v, w) and after the projection
    (u_proj, v_proj, w_proj), x fastest."""
    pos = np.ascontiguousarray(pos, np.float32).copy()
    vel = np.ascontiguousarray(vel, np.float32).copy()
    nc = P.nx * P.ny * P.nz
    u, v, w, phi, uq, vq, wq = (np.empty(nc, np.float64) for _ in range(7))
    info = NatInfo()
    sp = None
    if solid is not None:
        solid = np.ascontiguousarray(solid, np.uint8)
        sp = solid.ctypes.data
    lib().orc_nat_step_ex(pos.shape[0], pos, vel, sp, C.byref(P), u, v, w, phi, uq, vq, wq, C.byref(info))
    return dict(pos=pos, vel=vel, u=u, v=v, w=w, phi=phi, u_proj=uq, v_proj=vq, w_proj=wq, iters=info.iters,
                rel_residual=info.rel_residual, fluid_cells=info.fluid_cells)


def nat_pcg(type_, b, P):
    x = np.zeros(b.size, np.float64)
    rr = C.c_double(0.0)
    it = lib().orc_nat_pcg(np.ascontiguousarray(type_, np.uint8), np.ascontiguousarray(b, np.float64), x, C.byref(P), C.byref(rr))
    return x, it, rr.value


def nat_apply_A(type_, x, P):
    y = np.empty(x.size, np.float64)
    lib().orc_nat_apply_A(np.ascontiguousarray(type_, np.uint8), np.ascontiguousarray(x, np.float64), y, C.byref(P))
    return y


LP_DIL = (1, 2, 4, 1)


def lp_forward(type_, r, w, shape, dil=LP_DIL, round_bf16=True):
    """z = s N(r) of the learned preconditioner; shape (nx, ny, nz), arrays x fastest."""
    nx, ny, nz = shape
    z = np.empty(nx * ny * nz, np.float32)
    inv_s = C.c_double(0.0)
    lib().orc_lp_forward(nx, ny, nz, np.ascontiguousarray(type_, np.uint8).ravel(), np.ascontiguousarray(r, np.float32).ravel(),
                         np.ascontiguousarray(w, np.float32), np.ascontiguousarray(dil, np.int32), int(round_bf16), z,
                         C.byref(inv_s))
    return z, inv_s.value


def lp_loss_grad(type_, r, e, w, shape, dil=LP_DIL, round_bf16=True):
    """(loss, z = N(r), dloss/dw) of the A-norm loss of M(r) = N(r) + D^-1 r
    against the error e (A e = r): (m.Am - 2 m.r) / e.r + 1."""
    nx, ny, nz = shape
    z = np.empty(nx * ny * nz, np.float32)
    g = np.empty(lib().orc_lp_num_weights(), np.float64)
    loss = lib().orc_lp_loss_grad(nx, ny, nz, np.ascontiguousarray(type_, np.uint8).ravel(),
                                  np.ascontiguousarray(r, np.float32).ravel(), np.ascontiguousarray(e, np.float32).ravel(),
                                  np.ascontiguousarray(w, np.float32), np.ascontiguousarray(dil, np.int32), int(round_bf16),
                                  z, g)
    return loss, z, g


def lp_fpcg(type_, b, w, shape, tol=1e-6, max_iter=1000, dil=LP_DIL, round_bf16=True):
    """Flexible PCG with the network as preconditioner: (x, iterations, relative residual)."""
    nx, ny, nz = shape
    x = np.zeros(nx * ny * nz, np.float64)
    rr = C.c_double(0.0)
    it = lib().orc_lp_fpcg(nx, ny, nz, np.ascontiguousarray(type_, np.uint8).ravel(), np.ascontiguousarray(b, np.float64).ravel(),
                           np.ascontiguousarray(w, np.float32), np.ascontiguousarray(dil, np.int32), int(round_bf16), tol,
                           max_iter, x, C.byref(rr))
    return x, it, rr.value


def mg_levels(shape):
    """Padded (nx, ny, nz) of each level of the multilevel preconditioner."""
    dims = np.zeros(3 * 8, np.int32)
    n = lib().orc_mg_levels(shape[0], shape[1], shape[2], dims)
    return [tuple(int(v) for v in dims[3 * l:3 * l + 3]) for l in range(n)]


def mg_apply(type_, r, w, shape, mode=0, dil=LP_DIL, round_bf16=True):
    """One V-cycle z = M(r) of the multilevel preconditioner (FP64 apart from the network)."""
    nx, ny, nz = shape
    z = np.empty(nx * ny * nz, np.float64)
    lib().orc_mg_apply(nx, ny, nz, np.ascontiguousarray(type_, np.uint8).ravel(), np.ascontiguousarray(r, np.float32).ravel(),
                       np.ascontiguousarray(w, np.float32), np.ascontiguousarray(dil, np.int32), int(round_bf16), int(mode), z)
    return z


def mg_fcg(type_, b, w, shape, mode=0, tol=1e-6, max_iter=1000, dil=LP_DIL, round_bf16=True):
    """FCG with the multilevel preconditioner: (x, iterations, relative residual)."""
    nx, ny, nz = shape
    x = np.zeros(nx * ny * nz, np.float64)
    rr = C.c_double(0.0)
    it = lib().orc_mg_fcg(nx, ny, nz, np.ascontiguousarray(type_, np.uint8).ravel(), np.ascontiguousarray(b, np.float64).ravel(),
                          np.ascontiguousarray(w, np.float32), np.ascontiguousarray(dil, np.int32), int(round_bf16), int(mode),
                          tol, max_iter, x, C.byref(rr))
    return x, it, rr.value
