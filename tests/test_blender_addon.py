"""The Blender add-on (flip2_b200/blender_addon.py), which fills in the
reference's no-op FLUID SOLVER operator (plugin/plugin.py:22-27) with calls of
the C ABI, imported under a stand-in bpy.  Without a GPU the library calls go
to a recorder that checks the call sequence the operator makes; the GPU test
runs the operator on the real library."""
import ctypes as C
import importlib
import sys

import numpy as np
import pytest

from tests import fake_bpy


@pytest.fixture
def addon():
    bpy = fake_bpy.install()
    sys.modules.pop("flip2_b200.blender_addon", None)
    mod = importlib.import_module("flip2_b200.blender_addon")
    mod._velocities.clear()
    yield mod, bpy
    sys.modules.pop("flip2_b200.blender_addon", None)
    sys.modules.pop("bpy", None)


class RecordingLib:
    """Stands in for libflip2_b200.so: records each call, and on download
    moves every particle down by 0.01 and gives it velocity -1 in y."""

    def __init__(self):
        self.calls = []
        self.n = 0
        self.pos = None

    def __getattr__(self, name):
        def call(*args):
            self.calls.append(name)
            return self._do(name, args)
        return call

    def _do(self, name, args):
        if name == "flip_create":
            self.n = args[0]
            args[3]._obj.value = 1234
        elif name == "flip_upload_particles_f32":
            self.pos = [np.ctypeslib.as_array(C.cast(a, C.POINTER(C.c_float)), (self.n,)).copy() for a in args[1:4]]
        elif name == "flip_download_particles_f32":
            outs = [np.ctypeslib.as_array(C.cast(a, C.POINTER(C.c_float)), (self.n,)) for a in args[1:7]]
            for k in range(3):
                outs[k][:] = self.pos[k] - (0.01 if k == 1 else 0.0)
                outs[3 + k][:] = -1.0 if k == 1 else 0.0
        elif name in ("flip_last_error", "flip_status_string"):
            return b""
        return 0


def test_register_adds_the_operator_and_menu_entry(addon):
    mod, bpy = addon
    mod.register()
    assert bpy.registered == [mod.FluidSolver]
    assert bpy.types.VIEW3D_MT_object.items == [mod.menu_func]
    assert mod.FluidSolver.bl_idname == "fluid.solver"
    assert mod.bl_info["name"] == "FLUID SOLVER"
    mod.unregister()
    assert bpy.registered == [] and bpy.types.VIEW3D_MT_object.items == []


def test_execute_call_sequence_and_write_back(addon, monkeypatch):
    mod, bpy = addon
    lib = RecordingLib()
    monkeypatch.setattr(mod, "_lib", lambda: lib)
    pts = np.random.default_rng(0).uniform(0.2, 0.4, size=(100, 3)).astype(np.float32)
    fluid = fake_bpy.Object("Fluid", pts)
    other = fake_bpy.Object("Cube", np.zeros((8, 3)), fluid=False)
    scene = fake_bpy.Scene([fluid, other], fps=30, flip_domain=(0.0, 0.0, 0.0, 16, 1.0 / 16))
    op = mod.FluidSolver()
    assert op.execute(type("Ctx", (), {"scene": scene})()) == {"FINISHED"}
    assert lib.calls == ["flip_default_params", "flip_create", "flip_set_domain", "flip_upload_particles_f32",
                         "flip_initialize", "flip_solve_frame", "flip_download_particles_f32", "flip_destroy"]
    assert np.allclose(fluid.data.vertices.co[:, 1], pts[:, 1] - 0.01)
    assert np.array_equal(other.data.vertices.co, np.zeros((8, 3), np.float32))
    assert fluid.data.updates == 1
    # the velocities come back into the next frame's upload
    lib.calls.clear()
    op.execute(type("Ctx", (), {"scene": scene})())
    assert np.all(mod._velocities["Fluid"][:, 1] == -1.0)


def test_execute_reports_a_failing_call(addon, monkeypatch):
    mod, bpy = addon
    lib = RecordingLib()
    lib._do = lambda name, args: 7 if name == "flip_create" else (b"" if name in ("flip_last_error",
                                                                                 "flip_status_string") else 0)
    monkeypatch.setattr(mod, "_lib", lambda: lib)
    scene = fake_bpy.Scene([fake_bpy.Object("Fluid", np.full((4, 3), 0.5))])
    op = mod.FluidSolver()
    assert op.execute(type("Ctx", (), {"scene": scene})()) == {"CANCELLED"}
    assert op.reports and "flip_create" in op.reports[0][1]


@pytest.mark.gpu
def test_execute_on_the_library(addon):
    """The operator on libflip2_b200.so: a block of fluid falls for a frame."""
    mod, bpy = addon
    from flip2_b200 import scenes
    pos, _ = scenes.dam_break(32, seed=0)
    fluid = fake_bpy.Object("Fluid", pos)
    scene = fake_bpy.Scene([fluid], fps=24, flip_domain=(0.0, 0.0, 0.0, 8, 0.125))
    op = mod.FluidSolver()
    assert op.execute(type("Ctx", (), {"scene": scene})()) == {"FINISHED"}, getattr(op, "reports", None)
    out = fluid.data.vertices.co
    assert out.shape == pos.shape and np.all(np.isfinite(out))
    assert out[:, 1].mean() < pos[:, 1].mean()
    assert mod._velocities["Fluid"][:, 1].mean() < 0.0
