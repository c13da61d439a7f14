"""A stand-in for Blender's bpy module (absent here): just the pieces the
add-on in flip2_b200/blender_addon.py touches -- Operator, register_class,
the object menu, and scenes of mesh objects whose vertices support
foreach_get/foreach_set("co", ...)."""
import sys
import types

import numpy as np


class Operator:
    def report(self, kind, msg):
        self.reports = getattr(self, "reports", []) + [(set(kind), msg)]


class Menu:
    def __init__(self):
        self.items = []

    def append(self, f):
        self.items.append(f)

    def remove(self, f):
        self.items.remove(f)


class Vertices:
    def __init__(self, co):
        self.co = np.asarray(co, np.float32).reshape(-1, 3).copy()

    def __len__(self):
        return self.co.shape[0]

    def foreach_get(self, attr, out):
        assert attr == "co"
        out[:] = self.co.ravel()

    def foreach_set(self, attr, values):
        assert attr == "co"
        self.co = np.asarray(values, np.float32).reshape(-1, 3).copy()


class Mesh:
    def __init__(self, co):
        self.vertices = Vertices(co)
        self.updates = 0

    def update(self):
        self.updates += 1


class Object(dict):
    def __init__(self, name, co, fluid=True, type_="MESH"):
        super().__init__(flip_fluid=fluid)
        self.name = name
        self.type = type_
        self.data = Mesh(co)


class Scene(dict):
    def __init__(self, objects, fps=24, **props):
        super().__init__(**props)
        self.objects = objects
        self.render = types.SimpleNamespace(fps=fps)


def install():
    """Put a fresh stand-in bpy into sys.modules and return it."""
    bpy = types.ModuleType("bpy")
    bpy.registered = []
    bpy.types = types.SimpleNamespace(Operator=Operator, VIEW3D_MT_object=Menu())
    bpy.utils = types.SimpleNamespace(register_class=bpy.registered.append, unregister_class=bpy.registered.remove)
    sys.modules["bpy"] = bpy
    return bpy
