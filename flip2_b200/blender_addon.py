"""Blender add-on: the reference's FLUID SOLVER operator (plugin/plugin.py:8-39)
with its empty execute() filled in.  Like the reference add-on, which loads
libparticles.so with ctypes (plugin/plugin.py:4-5), it drives
libflip2_b200.so through its C ABI (include/flip2_b200.h) -- the calls below
are the ones a maintainer adds to plugin.py.

Scene contract (custom properties; all optional):
  object["flip_fluid"] = True    a mesh whose vertices are the particles (a
                                 point cloud: vertex order follows the
                                 engine's particle order after each frame)
  scene["flip_domain"] = (negX, negY, negZ, cells, cellSize)
                                 the reference's setDomain arguments with the
                                 same count on every axis; default the unit
                                 box as 64 root cells of 1/64 (256^3 voxels)
  scene["flip_mode"] = "native" or "reference"   (default "native")

Each execute() advances every fluid object by one frame at
scene.render.fps: the vertex coordinates (object space) are uploaded as
particle positions, with the velocities this add-on kept from the object's
previous frame (zero the first time), one flip_solve_frame runs, and the new
positions are written back into the mesh.
"""
import ctypes as C

import numpy as np

import bpy

bl_info = {
    "name": "FLUID SOLVER",
    "blender": (2, 80, 0),
    "category": "Object",
}

MODE_REFERENCE, MODE_NATIVE = 0, 1
DEFAULT_DOMAIN = (0.0, 0.0, 0.0, 64, 1.0 / 64.0)

# particle velocities carried between frames, per object name
_velocities = {}


def _lib():
    """libflip2_b200.so with its prototypes declared (flip2_b200.lib())."""
    from flip2_b200 import lib
    return lib()


class FlipError(RuntimeError):
    pass


def _check(L, rc, what, handle=None):
    if rc != 0:
        msg = L.flip_last_error(handle) or b""
        raise FlipError("%s failed: %s (%s)" % (what, L.flip_status_string(rc).decode(), msg.decode()))


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


def simulate_frame(L, points, velocities, fps, domain=DEFAULT_DOMAIN, mode=MODE_NATIVE):
    """One frame of the fluid: points and velocities (n, 3) float32 in and
    out, through the C ABI.  Returns (points, velocities) in the engine's
    particle order."""
    n = points.shape[0]
    px, py, pz = (np.ascontiguousarray(points[:, a], np.float32) for a in range(3))
    vx, vy, vz = (np.ascontiguousarray(velocities[:, a], np.float32) for a in range(3))
    params = _params_struct()()
    L.flip_default_params(mode, C.byref(params))
    h = C.c_void_p()
    _check(L, L.flip_create(n, C.byref(params), None, C.byref(h)), "flip_create")
    try:
        negx, negy, negz, cells, size = domain
        _check(L, L.flip_set_domain(h, negx, negy, negz, int(cells), int(cells), int(cells), size), "flip_set_domain", h)
        _check(L, L.flip_upload_particles_f32(h, _ptr(px), _ptr(py), _ptr(pz), _ptr(vx), _ptr(vy), _ptr(vz), n),
               "flip_upload_particles_f32", h)
        _check(L, L.flip_initialize(h), "flip_initialize", h)
        _check(L, L.flip_solve_frame(h, float(fps)), "flip_solve_frame", h)
        _check(L, L.flip_download_particles_f32(h, _ptr(px), _ptr(py), _ptr(pz), _ptr(vx), _ptr(vy), _ptr(vz), n),
               "flip_download_particles_f32", h)
    finally:
        L.flip_destroy(h)
    return np.stack([px, py, pz], 1), np.stack([vx, vy, vz], 1)


def _params_struct():
    from flip2_b200 import Params
    return Params


class FluidSolver(bpy.types.Operator):
    """Fluid Solver"""
    bl_idname = "fluid.solver"
    bl_label = "Simulate fluid motion of particles"
    bl_options = {'REGISTER', 'UNDO'}

    def execute(self, context):
        scene = context.scene
        fps = scene.render.fps
        domain = tuple(scene.get("flip_domain", DEFAULT_DOMAIN))
        mode = MODE_REFERENCE if scene.get("flip_mode", "native") == "reference" else MODE_NATIVE
        try:
            L = _lib()
            for obj in scene.objects:
                if obj.type != 'MESH' or not obj.get("flip_fluid", False):
                    continue
                verts = obj.data.vertices
                n = len(verts)
                if n == 0:
                    continue
                co = np.empty(3 * n, np.float32)
                verts.foreach_get("co", co)
                vel = _velocities.get(obj.name)
                if vel is None or vel.shape[0] != n:
                    vel = np.zeros((n, 3), np.float32)
                pts, vel = simulate_frame(L, co.reshape(n, 3), vel, fps, domain, mode)
                verts.foreach_set("co", np.ascontiguousarray(pts, np.float32).ravel())
                obj.data.update()
                _velocities[obj.name] = vel
        except (FlipError, OSError, RuntimeError) as err:
            self.report({'ERROR'}, str(err))
            return {'CANCELLED'}
        return {'FINISHED'}


def menu_func(self, context):
    self.layout.operator(FluidSolver.bl_idname)


def register():
    bpy.utils.register_class(FluidSolver)
    bpy.types.VIEW3D_MT_object.append(menu_func)


def unregister():
    bpy.utils.unregister_class(FluidSolver)
    bpy.types.VIEW3D_MT_object.remove(menu_func)


if __name__ == "__main__":
    register()
