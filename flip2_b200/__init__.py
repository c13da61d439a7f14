"""flip2_b200 -- a B200 (sm_100a) PIC/FLIP fluid step behind the flip2 engine API.

The compute lives in libflip2_b200.so (flip2_b200/lib/, built by
flip2_b200/build.py); this module binds its C ABI (include/flip2_b200.h) with
ctypes, the way the reference's Blender add-on loads libparticles.so
(plugin/plugin.py:4-5), and offers:

  * Particles -- the reference's engine class (engine/particles.hu:11-95)
    with the same method names, backed by a flip_engine handle;
  * primitives on torch CUDA tensors (ref_keys, sort_pairs, inclusive_scan,
    segment_heads, ...), each a thin call of one C entry point.

There is no CPU path: if the library is missing or no GPU is visible the calls
raise.
"""
import ctypes as C
import os

import numpy as np

from . import scenes  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libflip2_b200.so")
_LIB = None

MODE_REFERENCE = 0
MODE_NATIVE = 1

FLIP_OK = 0
STATUS = {0: "ok", 1: "bad argument", 2: "CUDA error", 3: "out of device memory", 4: "bounded device wait timed out",
          5: "call out of order", 6: "pressure solve did not converge", 7: "no usable device"}

# flip_buffer ids
(BUF_PX, BUF_PY, BUF_PZ, BUF_VX, BUF_VY, BUF_VZ, BUF_KEYS, BUF_PERM, BUF_FLAGS, BUF_STARTS, BUF_YTABLE,
 BUF_NODE_VOXELS, BUF_VOXEL_IDS, BUF_SOLIDS, BUF_UX, BUF_UY, BUF_UZ, BUF_DIVU, BUF_P, BUF_RES,
 BUF_GRID_U, BUF_GRID_V, BUF_GRID_W, BUF_CELL_TYPE, BUF_PRESSURE, BUF_TILE_LIST,
 BUF_GRID_U_P2G, BUF_GRID_V_P2G, BUF_GRID_W_P2G,
 BUF_MG_COARSE_TYPE, BUF_MG_COARSE_R, BUF_MG_COARSE_E) = range(32)


class FlipError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("flip2_b200: %s (%d): %s" % (STATUS.get(status, "?"), status, msg))
        self.status = status


class Grid(C.Structure):
    """Field for field the reference's Grid (engine/grid.hpp:8-38)."""
    _fields_ = [("negX", C.c_float), ("negY", C.c_float), ("negZ", C.c_float),
                ("sizeX", C.c_uint32), ("sizeY", C.c_uint32), ("sizeZ", C.c_uint32),
                ("cellSize", C.c_float)]


class Params(C.Structure):
    _fields_ = [("mode", C.c_int32), ("flip_ratio", C.c_float), ("gravity_y", C.c_float), ("pcg_tol", C.c_double),
                ("pcg_max_iter", C.c_int32), ("pcg_check_every", C.c_int32), ("true_residual_every", C.c_int32),
                ("permute_velocities", C.c_int32), ("device", C.c_int32), ("pressure_method", C.c_int32),
                ("max_substep_dt", C.c_double), ("learned_max_iter", C.c_int32), ("lp_cuda_cores", C.c_int32),
                ("pcg_warm_start", C.c_int32), ("mg_coarse", C.c_int32)]


class PoissonSpec(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("surface_min", C.c_double), ("surface_max", C.c_double),
                ("solid_fraction", C.c_double), ("radius_min", C.c_double), ("radius_max", C.c_double),
                ("impulses", C.c_int32), ("reserved", C.c_int32), ("gravity_dt", C.c_double)]


class SolveInfo(C.Structure):
    _fields_ = [("iters", C.c_int32), ("converged", C.c_int32), ("fell_back", C.c_int32), ("plain_iters", C.c_int32),
                ("rel_residual", C.c_double), ("ms", C.c_double)]


class Info(C.Structure):
    _fields_ = [("nodes", C.c_uint32), ("voxels", C.c_uint32), ("pressure_iters", C.c_int32), ("converged", C.c_int32),
                ("dt", C.c_double), ("residual", C.c_double), ("elapsed_time", C.c_double), ("n", C.c_uint64),
                ("error_flags", C.c_uint32), ("launches", C.c_uint32), ("solves", C.c_uint64),
                ("fallbacks", C.c_uint64), ("pressure_iters_total", C.c_uint64), ("graph_steps", C.c_uint64)]


def lib():
    """Load libflip2_b200.so and declare its prototypes (raises if absent)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libflip2_b200.so is not built; run `python flip2_b200/build.py` (or __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    vp, u64, u32, i32, d, sz = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int, C.c_double, C.c_size_t
    gp = C.POINTER(Grid)
    protos = {
        "flip_version": (C.c_char_p, []),
        "flip_status_string": (C.c_char_p, [i32]),
        "flip_ref_keys": (i32, [vp, vp, vp, u64, gp, vp, vp, vp]),
        "flip_sort_pairs_scratch_bytes": (sz, [u64]),
        "flip_sort_pairs": (i32, [vp, vp, vp, vp, u64, i32, vp, sz, vp]),
        "flip_inclusive_scan_scratch_bytes": (sz, [u64]),
        "flip_inclusive_scan_u32": (i32, [vp, vp, u64, vp, sz, vp]),
        "flip_inclusive_scan_u32_noalloc": (i32, [vp, vp, u64, vp]),
        "flip_inclusive_scan_u32_noalloc_status": (i32, [vp, C.POINTER(u32)]),
        "flip_scratch_status": (i32, [vp, vp, C.POINTER(u32)]),
        "flip_test_lookback_timeout": (i32, [i32, vp, vp, vp, u64, u32, vp, sz, vp, C.POINTER(u32)]),
        "flip_binary_version": (i32, [C.POINTER(i32)]),
        "flip_segment_heads_scratch_bytes": (sz, [u64]),
        "flip_segment_heads": (i32, [vp, u64, vp, vp, vp, vp, vp, sz, vp]),
        "flip_ref_ydim_rows": (i32, [vp, vp, u32, gp, vp, vp]),
        "flip_ref_voxel_counts": (i32, [vp, vp, u32, u64, vp, vp, vp, gp, vp, vp, vp]),
        "flip_ref_voxel_ids": (i32, [vp, u32, vp, vp, gp, vp, vp, vp]),
        "flip_ref_p2g": (i32, [vp, vp, u32, u64, vp, vp, vp, vp, vp, vp, vp, vp, vp, gp, vp, vp, vp, vp]),
        "flip_ref_g2p": (i32, [vp, vp, u32, u64, vp, vp, vp, vp, vp, vp, vp, vp, gp, vp, vp, vp, vp]),
        "flip_ref_getmax_scratch_bytes": (sz, [u64]),
        "flip_ref_getmax_f64": (i32, [vp, u64, i32, vp, sz, C.POINTER(d), vp]),
        "flip_default_params": (None, [i32, C.POINTER(Params)]),
        "flip_create": (i32, [u64, C.POINTER(Params), vp, C.POINTER(vp)]),
        "flip_set_domain": (i32, [vp, d, d, d, u32, u32, u32, d]),
        "flip_upload_particles_f64": (i32, [vp, vp, vp, vp, vp, vp, vp, u64]),
        "flip_download_particles_f64": (i32, [vp, vp, vp, vp, vp, vp, vp, u64]),
        "flip_upload_particles_f32": (i32, [vp, vp, vp, vp, vp, vp, vp, u64]),
        "flip_download_particles_f32": (i32, [vp, vp, vp, vp, vp, vp, vp, u64]),
        "flip_set_solid_mask": (i32, [vp, vp, u64]),
        "flip_align_particles_to_grid": (i32, [vp]),
        "flip_sort_particles": (i32, [vp]),
        "flip_generate_voxels": (i32, [vp]),
        "flip_particle_vel_to_voxels": (i32, [vp]),
        "flip_pressure_solve": (i32, [vp]),
        "flip_update_voxel_velocities": (i32, [vp]),
        "flip_voxel_vels_to_particles": (i32, [vp]),
        "flip_advect_particles": (i32, [vp]),
        "flip_move_solid_particles": (i32, [vp]),
        "flip_initialize": (i32, [vp]),
        "flip_solve_frame": (i32, [vp, d]),
        "flip_get_courant_dt": (d, [vp]),
        "flip_write_positions_csv": (i32, [vp, C.c_char_p]),
        "flip_write_positions_bin": (i32, [vp, C.c_char_p]),
        "flip_step_streamed_f32": (i32, [vp] * 7 + [u64, d]),
        "flip_set_solid_velocity": (i32, [vp, d, d, d]),
        "flip_step": (i32, [vp, d]),
        "flip_sync": (i32, [vp]),
        "flip_get_buffer": (i32, [vp, i32, C.POINTER(vp), C.POINTER(u64), C.POINTER(u32)]),
        "flip_read_buffer": (i32, [vp, i32, vp, u64]),
        "flip_get_info": (i32, [vp, C.POINTER(Info)]),
        "flip_get_solve_info": (i32, [vp, C.POINTER(SolveInfo)]),
        "flip_lp_num_weights": (u64, []),
        "flip_lp_init": (i32, [vp, u64]),
        "flip_lp_set_weights": (i32, [vp, vp, u64]),
        "flip_lp_get_weights": (i32, [vp, vp, u64]),
        "flip_lp_get_grad": (i32, [vp, vp, u64]),
        "flip_poisson_generate": (i32, [vp, C.POINTER(PoissonSpec)]),
        "flip_poisson_set": (i32, [vp, vp, vp]),
        "flip_poisson_solve": (i32, [vp, i32, d, i32, C.POINTER(SolveInfo)]),
        "flip_poisson_read_solution": (i32, [vp, vp]),
        "flip_lp_train_step": (i32, [vp, i32, C.c_float, C.POINTER(d)]),
        "flip_lp_eval": (i32, [vp, vp, vp, vp, C.POINTER(d), i32]),
        "flip_mg_apply": (i32, [vp, vp, vp]),
        "flip_mg_train_step": (i32, [vp, i32, C.c_float, C.POINTER(d)]),
        "flip_set_timing": (i32, [vp, i32]),
        "flip_get_stage_ms": (i32, [vp, C.POINTER(C.c_double), i32, i32]),
        "flip_last_error": (C.c_char_p, [vp]),
        "flip_destroy": (i32, [vp]),
    }
    for name, (res, args) in protos.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _LIB = L
    return L


def exported_symbols():
    """Names of the C entry points declared in include/flip2_b200.h."""
    import re
    hdr = os.path.join(os.path.dirname(_HERE), "include", "flip2_b200.h")
    text = open(hdr).read()
    return sorted(set(re.findall(r"\b(flip_[a-z0-9_]+)\s*\(", text)))


def _check(rc, what, engine=None):
    if rc != FLIP_OK:
        L = lib()
        msg = L.flip_last_error(engine) if engine is not None else L.flip_last_error(None)
        raise FlipError(rc, "%s: %s" % (what, (msg or b"").decode()))


def make_grid(negX, negY, negZ, X, Y, Z, cellSize):
    return Grid(negX, negY, negZ, X, Y, Z, cellSize)


def default_params(mode=MODE_NATIVE, **kw):
    p = Params()
    lib().flip_default_params(mode, C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


# ------------------------------------------------------------ primitives
def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _scratch(nbytes, device):
    import torch
    return torch.empty(max(int(nbytes), 16), dtype=torch.uint8, device=device)


def ref_keys(px, py, pz, grid, with_index=False, stream=None):
    """rootCell on FP64 CUDA tensors (clamped in place); returns keys (and iota)."""
    import torch
    n = px.numel()
    keys = torch.empty(n, dtype=torch.int32, device=px.device)
    idx = torch.empty(n, dtype=torch.int32, device=px.device) if with_index else None
    _check(lib().flip_ref_keys(_ptr(px), _ptr(py), _ptr(pz), n, C.byref(grid), _ptr(keys), _ptr(idx), _stream(stream)),
           "flip_ref_keys")
    return (keys, idx) if with_index else keys


def sort_pairs(keys, vals=None, key_bits=32, out_keys=None, out_vals=None, stream=None, return_scratch=False):
    """Stable radix sort of u32 keys (int32 tensors holding the bits); returns
    (sorted_keys, sorted_vals) where vals default to the index permutation."""
    import torch
    n = keys.numel()
    ok = out_keys if out_keys is not None else torch.empty_like(keys)
    ov = out_vals if out_vals is not None else torch.empty(n, dtype=torch.int32, device=keys.device)
    nb = lib().flip_sort_pairs_scratch_bytes(n)
    scr = _scratch(nb, keys.device)
    _check(lib().flip_sort_pairs(_ptr(keys), _ptr(vals), _ptr(ok), _ptr(ov), n, key_bits, _ptr(scr), nb, _stream(stream)),
           "flip_sort_pairs")
    if return_scratch:
        return ok, ov, scr
    return ok, ov


def inclusive_scan(x, out=None, stream=None, return_scratch=False):
    import torch
    n = x.numel()
    o = out if out is not None else torch.empty_like(x)
    nb = lib().flip_inclusive_scan_scratch_bytes(n)
    scr = _scratch(nb, x.device)
    _check(lib().flip_inclusive_scan_u32(_ptr(x), _ptr(o), n, _ptr(scr), nb, _stream(stream)), "flip_inclusive_scan_u32")
    if return_scratch:
        return o, scr
    return o


def segment_heads(sorted_keys, want_flags=True, want_keys=True, stream=None):
    """Returns (flags_scan or None, starts[:count], node_keys[:count] or None, count)."""
    import torch
    n = sorted_keys.numel()
    dev = sorted_keys.device
    flags = torch.empty(n, dtype=torch.int32, device=dev) if want_flags else None
    starts = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    nk = torch.empty(max(n, 1), dtype=torch.int32, device=dev) if want_keys else None
    cnt = torch.zeros(1, dtype=torch.int32, device=dev)
    nb = lib().flip_segment_heads_scratch_bytes(n)
    scr = _scratch(nb, dev)
    _check(lib().flip_segment_heads(_ptr(sorted_keys), n, _ptr(flags), _ptr(starts), _ptr(nk), _ptr(cnt), _ptr(scr), nb,
                                    _stream(stream)), "flip_segment_heads")
    c = int(cnt.item())
    return flags, starts[:c], (nk[:c] if nk is not None else None), c


def ref_ydim_rows(starts, sorted_keys, nodes, grid, stream=None):
    import torch
    table = torch.empty(grid.sizeY * grid.sizeZ, dtype=torch.int32, device=starts.device)
    _check(lib().flip_ref_ydim_rows(_ptr(starts), _ptr(sorted_keys), nodes, C.byref(grid), _ptr(table), _stream(stream)),
           "flip_ref_ydim_rows")
    return table


def ref_voxels(starts, sorted_keys, nodes, px, py, pz, grid, stream=None):
    """getNumberVoxelsUsedPerNode + scan + generateVoxelIDs; returns
    (counts, node_voxels, voxel_ids, solids)."""
    import torch
    dev = starts.device
    n = px.numel()
    counts = torch.empty(nodes, dtype=torch.int32, device=dev)
    masks = torch.empty(nodes * 16, dtype=torch.int32, device=dev)
    _check(lib().flip_ref_voxel_counts(_ptr(starts), _ptr(sorted_keys), nodes, n, _ptr(px), _ptr(py), _ptr(pz),
                                       C.byref(grid), _ptr(counts), _ptr(masks), _stream(stream)), "flip_ref_voxel_counts")
    node_voxels = inclusive_scan(counts, stream=stream)
    nvox = int(node_voxels[-1].item()) if nodes else 0
    ids = torch.empty(max(nvox, 1), dtype=torch.int32, device=dev)
    sol = torch.empty(max(nvox, 1), dtype=torch.int8, device=dev)
    _check(lib().flip_ref_voxel_ids(_ptr(sorted_keys), nodes, _ptr(masks), _ptr(node_voxels), C.byref(grid), _ptr(ids),
                                    _ptr(sol), _stream(stream)), "flip_ref_voxel_ids")
    return counts, node_voxels, ids[:nvox], sol[:nvox]


def ref_p2g(starts, sorted_keys, nodes, px, py, pz, vx, vy, vz, node_voxels, voxel_ids, solids, grid, stream=None):
    import torch
    nvox = voxel_ids.numel()
    out = [torch.empty(max(nvox, 1), dtype=torch.float64, device=px.device) for _ in range(3)]
    _check(lib().flip_ref_p2g(_ptr(starts), _ptr(sorted_keys), nodes, px.numel(), _ptr(px), _ptr(py), _ptr(pz), _ptr(vx),
                              _ptr(vy), _ptr(vz), _ptr(node_voxels), _ptr(voxel_ids), _ptr(solids), C.byref(grid),
                              _ptr(out[0]), _ptr(out[1]), _ptr(out[2]), _stream(stream)), "flip_ref_p2g")
    return [o[:nvox] for o in out]


def ref_g2p(starts, sorted_keys, nodes, px, py, pz, node_voxels, voxel_ids, ux, uy, uz, grid, stream=None):
    import torch
    n = px.numel()
    out = [torch.empty(n, dtype=torch.float64, device=px.device) for _ in range(3)]
    _check(lib().flip_ref_g2p(_ptr(starts), _ptr(sorted_keys), nodes, n, _ptr(px), _ptr(py), _ptr(pz), _ptr(node_voxels),
                              _ptr(voxel_ids), _ptr(ux), _ptr(uy), _ptr(uz), C.byref(grid), _ptr(out[0]), _ptr(out[1]),
                              _ptr(out[2]), _stream(stream)), "flip_ref_g2p")
    return out


# ------------------------------------------------------------ engine
_NP = {1: np.int8, 4: np.uint32, 8: np.float64}


class Particles:
    """The reference's Particles class (engine/particles.hu:11-95) over a
    flip_engine handle.  Method names follow the reference; state lives on the
    GPU and moves to the host only through upload/download/buffer reads."""

    def __init__(self, size, mode=MODE_NATIVE, params=None, stream=None):
        L = lib()
        p = params if params is not None else default_params(mode)
        p.mode = mode
        h = C.c_void_p()
        st = C.c_void_p(stream) if stream is not None else None
        _check(L.flip_create(size, C.byref(p), st, C.byref(h)), "flip_create")
        self._h = h
        self.size = size
        self.mode = mode
        self.params = p

    # lifetime
    def close(self):
        if getattr(self, "_h", None):
            lib().flip_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _call(self, name, *args):
        _check(getattr(lib(), name)(self._h, *args), name, self._h)

    # Particles API
    def setDomain(self, nx, ny, nz, x, y, z, cellSize):
        self._call("flip_set_domain", nx, ny, nz, x, y, z, cellSize)
        self.params_grid_cells = 64 * x * y * z

    def alignParticlesToGrid(self):
        self._call("flip_align_particles_to_grid")

    def sortParticles(self):
        self._call("flip_sort_particles")

    def generateVoxels(self):
        self._call("flip_generate_voxels")

    def particleVelToVoxels(self):
        self._call("flip_particle_vel_to_voxels")

    def pressureSolve(self):
        self._call("flip_pressure_solve")

    def updateVoxelVelocities(self):
        self._call("flip_update_voxel_velocities")

    def voxelVelsToParticles(self):
        self._call("flip_voxel_vels_to_particles")

    def advectParticles(self):
        self._call("flip_advect_particles")

    def moveSolidParticles(self):
        self._call("flip_move_solid_particles")

    def initialize(self):
        self._call("flip_initialize")

    def solveFrame(self, fps):
        self._call("flip_solve_frame", fps)

    def getCourantDt(self):
        return lib().flip_get_courant_dt(self._h)

    def writePositionsToFile(self, fileName):
        self._call("flip_write_positions_csv", str(fileName).encode())

    def write_positions_bin(self, fileName):
        self._call("flip_write_positions_bin", str(fileName).encode())

    # extensions
    def step(self, dt):
        self._call("flip_step", dt)

    def sync(self):
        self._call("flip_sync")

    def upload(self, pos, vel=None):
        """pos, vel: (n,3) arrays (float32 or float64) or tuples of 3 arrays."""
        def cols(a, dt):
            if a is None:
                return [None, None, None]
            if isinstance(a, (tuple, list)):
                return [np.ascontiguousarray(c, dt) for c in a]
            a = np.asarray(a)
            return [np.ascontiguousarray(a[:, k], dt) for k in range(3)]
        dt = np.float64 if self.mode == MODE_REFERENCE else np.float32
        P = cols(pos, dt)
        V = cols(vel, dt)
        n = P[0].size
        if any(c is not None and c.size != n for c in P + V):
            raise FlipError(1, "upload: position and velocity columns differ in length")
        ptrs = [c.ctypes.data_as(C.c_void_p) if c is not None else None for c in P + V]
        fn = "flip_upload_particles_f64" if dt == np.float64 else "flip_upload_particles_f32"
        self._call(fn, *ptrs, n)  # the engine rejects n != its size (FLIP_ERR_ARG)
        self._keep = P + V

    def upload_ptrs(self, ptrs, f64=False):
        """Upload from six host pointers (pinned or pageable), no copies in Python."""
        fn = "flip_upload_particles_f64" if f64 else "flip_upload_particles_f32"
        self._call(fn, *[C.c_void_p(p) if p else None for p in ptrs], self.size)

    def step_streamed(self, ptrs, dt):
        """Upload from six host float32 arrays (pointers), one step, download into
        them; returns before the download ends (sync() waits for it)."""
        self._call("flip_step_streamed_f32", *[C.c_void_p(p) for p in ptrs], self.size, dt)

    def download_ptrs(self, ptrs, f64=False):
        fn = "flip_download_particles_f64" if f64 else "flip_download_particles_f32"
        self._call(fn, *[C.c_void_p(p) if p else None for p in ptrs], self.size)

    def download(self, dtype=None):
        dt = dtype or (np.float64 if self.mode == MODE_REFERENCE else np.float32)
        out = [np.empty(self.size, dt) for _ in range(6)]
        fn = "flip_download_particles_f64" if dt == np.float64 else "flip_download_particles_f32"
        self._call(fn, *[o.ctypes.data_as(C.c_void_p) for o in out], self.size)
        return np.stack(out[:3], axis=1), np.stack(out[3:], axis=1)

    def set_solid_mask(self, mask):
        m = np.ascontiguousarray(mask, np.uint8)
        self._call("flip_set_solid_mask", m.ctypes.data_as(C.c_void_p), m.size)

    def set_solid_velocity(self, ux, uy, uz):
        self._call("flip_set_solid_velocity", ux, uy, uz)

    def buffer_ptr(self, which):
        p, c, es = C.c_void_p(), C.c_uint64(), C.c_uint32()
        self._call("flip_get_buffer", which, C.byref(p), C.byref(c), C.byref(es))
        return p.value, c.value, es.value

    def read(self, which, dtype=None):
        _, c, es = self.buffer_ptr(which)
        dt = dtype or _NP[es]
        out = np.empty(c * es // np.dtype(dt).itemsize, dt)
        if out.nbytes:
            self._call("flip_read_buffer", which, out.ctypes.data_as(C.c_void_p), out.nbytes)
        return out

    STAGES = ("keys", "sort", "gather", "segment_heads", "grid_clear", "p2g", "tile_dilation", "normalize_gravity",
              "pcg_setup", "pcg_iterations", "projection", "g2p_advect")

    def set_timing(self, on=True):
        self._call("flip_set_timing", 1 if on else 0)

    def stage_ms(self, reset=False):
        a = (C.c_double * len(self.STAGES))()
        self._call("flip_get_stage_ms", a, len(self.STAGES), 1 if reset else 0)
        return dict(zip(self.STAGES, list(a)))

    # learned preconditioner and standalone pressure problems
    def lp_init(self, seed=0):
        self._call("flip_lp_init", seed)

    def lp_weights(self):
        n = lib().flip_lp_num_weights()
        w = np.empty(n, np.float32)
        self._call("flip_lp_get_weights", w.ctypes.data_as(C.c_void_p), n)
        return w

    def lp_set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        self._call("flip_lp_set_weights", w.ctypes.data_as(C.c_void_p), w.size)

    def lp_grad(self):
        n = lib().flip_lp_num_weights()
        g = np.empty(n, np.float32)
        self._call("flip_lp_get_grad", g.ctypes.data_as(C.c_void_p), n)
        return g

    def poisson_generate(self, seed, surface=(0.5, 0.85), solid_fraction=0.10, radius=(4.0, 16.0), impulses=6,
                         gravity_dt=-9.8 / 480.0):
        spec = PoissonSpec(seed, surface[0], surface[1], solid_fraction, radius[0], radius[1], impulses, 0, gravity_dt)
        self._call("flip_poisson_generate", C.byref(spec))

    def poisson_set(self, type_lin, b_lin):
        t = np.ascontiguousarray(type_lin, np.uint8)
        b = np.ascontiguousarray(b_lin, np.float32)
        self._call("flip_poisson_set", t.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p))

    def poisson_solve(self, method=0, tol=1e-6, max_iter=10000):
        i = SolveInfo()
        self._call("flip_poisson_solve", method, tol, max_iter, C.byref(i))
        return i

    def solve_info(self):
        i = SolveInfo()
        self._call("flip_get_solve_info", C.byref(i))
        return i

    def poisson_solution(self):
        nc = int(self.params_grid_cells)
        x = np.empty(nc, np.float64)
        self._call("flip_poisson_read_solution", x.ctypes.data_as(C.c_void_p))
        return x

    def lp_train_step(self, sample, lr):
        """sample >= 0: Jacobi-PCG iterate error; -1: white-noise error."""
        loss = C.c_double()
        self._call("flip_lp_train_step", sample, lr, C.byref(loss))
        return loss.value

    def lp_eval(self, r_lin, e_lin, want_grad=False):
        r = np.ascontiguousarray(r_lin, np.float32)
        ev = np.ascontiguousarray(e_lin, np.float32)
        z = np.empty_like(r)
        loss = C.c_double()
        self._call("flip_lp_eval", r.ctypes.data_as(C.c_void_p), ev.ctypes.data_as(C.c_void_p),
                   z.ctypes.data_as(C.c_void_p), C.byref(loss), 1 if want_grad else 0)
        return z, loss.value

    def mg_apply(self, r_lin):
        """One V-cycle of the multilevel preconditioner, z = M(r), x fastest."""
        r = np.ascontiguousarray(r_lin, np.float32)
        z = np.empty_like(r)
        self._call("flip_mg_apply", r.ctypes.data_as(C.c_void_p), z.ctypes.data_as(C.c_void_p))
        return z

    def mg_train_step(self, sample, lr):
        """Train the network as the V-cycle's coarsest solve.  sample >= 0:
        the coarse right-hand side of the residual after that many Jacobi-PCG
        iterations; -1: white-noise coarse error."""
        loss = C.c_double()
        self._call("flip_mg_train_step", sample, lr, C.byref(loss))
        return loss.value

    def info(self):
        i = Info()
        self._call("flip_get_info", C.byref(i))
        return i


def read_positions_bin(path):
    """(n, 3) float32 positions of a frame written by flip_write_positions_bin."""
    with open(path, "rb") as f:
        head = f.read(16)
        if len(head) != 16 or head[:8] != b"FLIP2POS":
            raise ValueError("%s: not a FLIP2POS frame" % path)
        n = int(np.frombuffer(head[8:], np.uint64)[0])
        data = np.frombuffer(f.read(12 * n), np.float32)
    if data.size != 3 * n:
        raise ValueError("%s: truncated frame" % path)
    return data.reshape(n, 3)
