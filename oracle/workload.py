"""ORACLE (test infrastructure): a frame's scene and host side without the
product's library, for the CPU arm of the benchmark.

OracleSetup has the fields oracle/frame.py's FrameRunner reads from
tests.helpers.SceneSetup, built from:

  * the seeded procedural scene: oracle_mesh_procedural (the workload
    generator's source compiled into liboracle.so);
  * the BVH and the light list: the reference's own src/bvh.cpp and
    src/lights.cpp (oracle/_ref/libref_bvh.so);
  * the uniforms of each frame: oracle_frame_params, the oracle's
    restatement of renderer.cpp:435-731 (OracleHost).

Nothing here loads restir_b200's library: restir_b200.abi only defines the
ctypes structures.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from restir_b200.abi import (RestirBvhDesc, RestirDisplayParams, RestirFrameInput, RestirFramePlan,
                             RestirFrameState, RestirMeshDesc, RestirParams, RestirScene, RestirSettings)

from . import binding as ob

P = C.c_void_p
u32 = C.c_uint32

_HOST_SIGNATURES = {
    "oracle_settings_default": (None, [C.POINTER(RestirSettings)]),
    "oracle_frame_params": (C.c_int, [C.POINTER(RestirSettings), C.POINTER(RestirMeshDesc), u32,
                                      C.POINTER(RestirBvhDesc), C.POINTER(RestirFrameInput),
                                      C.POINTER(RestirFrameState), C.POINTER(RestirParams),
                                      C.POINTER(RestirFramePlan)]),
    "oracle_frame_advance": (None, [C.POINTER(RestirParams), C.POINTER(RestirFramePlan), C.POINTER(RestirFrameInput),
                                    C.POINTER(RestirFrameState)]),
    "oracle_display_params": (C.c_int, [P, P, u32, u32, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                        C.c_float, C.c_int, C.c_int, C.c_int, C.POINTER(RestirDisplayParams)]),
    "oracle_mesh_procedural": (P, [C.c_int, u32, u32]),
    "oracle_mesh_describe": (C.c_int, [P, C.POINTER(RestirMeshDesc)]),
    "oracle_mesh_destroy": (None, [P]),
}


def lib():
    library = ob.load()
    if not getattr(library, "_host_bound", False):
        for name, (restype, argtypes) in _HOST_SIGNATURES.items():
            fn = getattr(library, name)
            fn.restype = restype
            fn.argtypes = argtypes
        library._host_bound = True
    return library


def check(status: int, what: str) -> None:
    if status != 0:
        raise RuntimeError(f"{what} failed with status {status}")


class OracleHost:
    """The host side of a frame through the oracle (oracle_frame.cpp)."""

    def frame_params(self, settings, mesh, light_count, bvh, frame_input, state):
        params, plan = RestirParams(), RestirFramePlan()
        check(lib().oracle_frame_params(C.byref(settings), C.byref(mesh.desc), light_count, C.byref(bvh.desc),
                                        C.byref(frame_input), C.byref(state), C.byref(params), C.byref(plan)),
              "oracle_frame_params")
        return params, plan

    def advance(self, params, plan, frame_input, state):
        lib().oracle_frame_advance(C.byref(params), C.byref(plan), C.byref(frame_input), C.byref(state))

    def display_params(self, *args):
        out = RestirDisplayParams()
        check(lib().oracle_display_params(*args, C.byref(out)), "oracle_display_params")
        return out


class OracleMesh:
    """A seeded procedural scene (RESTIR_SCENE_*), with the product's Mesh fields."""

    def __init__(self, kind: int, seed: int = 0, triangles: int = 0):
        self.handle = lib().oracle_mesh_procedural(kind, seed, triangles)
        if not self.handle:
            raise RuntimeError("oracle_mesh_procedural failed")
        self.desc = RestirMeshDesc()
        check(lib().oracle_mesh_describe(self.handle, C.byref(self.desc)), "oracle_mesh_describe")

    @property
    def triangle_count(self) -> int:
        return self.desc.triangle_count

    def array(self, field: str, ctype, count: int) -> np.ndarray:
        pointer = getattr(self.desc, field)
        return np.ctypeslib.as_array(C.cast(pointer, C.POINTER(ctype)), (count,)).copy() if pointer else None

    def __del__(self):
        if getattr(self, "handle", None):
            lib().oracle_mesh_destroy(self.handle)
            self.handle = None


class OracleBvh:
    """The reference builder's buffer (src/bvh.cpp) for a mesh, with the
    per-slot shading normals the ray-cast G-buffer reads: each slot's
    triangle is found among the mesh's by its three vertices (the builder
    copies them exactly)."""

    def __init__(self, mesh: OracleMesh):
        n = mesh.triangle_count
        positions = mesh.array("positions", C.c_float, 9 * n).reshape(n, 9)
        triangle_material = mesh.array("triangle_material", C.c_uint32, n)
        materials = mesh.array("materials", C.c_float, 8 * mesh.desc.material_count).reshape(-1, 8)
        normals = mesh.array("normals", C.c_float, 3 * n).reshape(n, 3)
        two_sided = mesh.array("two_sided", C.c_uint8, n)
        self.data, node_count, offset, depth = ob.reference_bvh(positions, triangle_material, materials)
        rows = self.data[4 * offset:].reshape(n, 4, 4)
        slot_positions = np.ascontiguousarray(rows[:, 0:3, 0:3].reshape(n, 9))
        self.order = _match_rows(slot_positions, positions)
        self.triangle_normals = np.zeros((n, 4), np.float32)
        self.triangle_normals[:, 0:3] = normals[self.order]
        if two_sided is not None:
            self.triangle_normals[:, 3] = two_sided[self.order]
        self.triangle_normals = self.triangle_normals.reshape(-1)
        self.desc = RestirBvhDesc()
        self.desc.node_count, self.desc.triangle_offset, self.desc.triangle_count = node_count, offset, n
        self.depth = depth


def _match_rows(rows: np.ndarray, table: np.ndarray) -> np.ndarray:
    """For each row of `rows`, the index of a bit-identical row of `table`."""
    key = np.dtype((np.void, rows.dtype.itemsize * rows.shape[1]))
    a = np.ascontiguousarray(rows).view(key).ravel()
    b = np.ascontiguousarray(table).view(key).ravel()
    order = np.argsort(b, kind="stable")
    found = np.searchsorted(b[order], a)
    index = order[np.minimum(found, len(b) - 1)]
    if not np.array_equal(b[index], a):
        raise RuntimeError("a BVH triangle matches no mesh triangle")
    return index.astype(np.uint32)


class OracleLights:
    """The reference's light list (src/lights.cpp) over the last OracleBvh's
    emitters and the seeded extra point lights."""

    def __init__(self, mesh: OracleMesh, settings: RestirSettings):
        if not settings.emissive_lighting:
            raise RuntimeError("the oracle's scene set-up keeps the emitters in the light list")
        scale = (mesh.desc.radius / 1.75) ** 2
        self.data, self.count, self.triangles = ob.reference_lights(
            settings.extra_lights, settings.extra_intensity, settings.extra_seed, list(mesh.desc.bounds_min),
            list(mesh.desc.bounds_max), scale)
        if self.count == 0:
            self.data = np.zeros(16, np.float32)


class OracleSetup:
    """tests.helpers.SceneSetup's fields, without the product's library."""

    def __init__(self, kind: int, seed: int = 0, triangles: int = 0, extra_lights: int = 0):
        self.mesh = OracleMesh(kind, seed, triangles)
        self.settings = RestirSettings()
        lib().oracle_settings_default(C.byref(self.settings))
        for k in range(3):
            self.settings.light_position[k] = self.mesh.desc.light_position[k]
        self.settings.sky_enabled = self.mesh.desc.sky
        self.settings.extra_lights = extra_lights
        self.bvh = OracleBvh(self.mesh)
        self.lights = OracleLights(self.mesh, self.settings)
        self.materials = self.mesh.array("materials", C.c_float, 8 * self.mesh.desc.material_count).reshape(-1, 8)
        self.host_side = OracleHost()

    def host_scene(self) -> RestirScene:
        s = RestirScene()
        s.bvh = self.bvh.data.ctypes.data
        s.node_count = self.bvh.desc.node_count
        s.triangle_offset = self.bvh.desc.triangle_offset
        s.triangle_count = self.bvh.desc.triangle_count
        s.lights = self.lights.data.ctypes.data
        s.light_count = self.lights.count
        s.triangle_normals = self.bvh.triangle_normals.ctypes.data
        s.materials = self.materials.ctypes.data
        s.material_count = len(self.materials)
        return s
