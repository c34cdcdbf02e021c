"""restir-b200: B200-native per-frame light transport of the pkonecki/restir renderer.

The product is librestir_gpu.so (hand-written sm_100a CUDA kernels behind the
C ABI of include/restir_gpu.h, and the C++ frame driver and scene preparation
of include/restir_frame.h and include/restir_host.h). This module loads it
through ctypes and mirrors the reference renderer's interface
(src/renderer.h:73-125: init, setScene, render, invalidateHistory,
setReferenceAccumulation, frameSubmitted / metrics) for Python callers.

There is no CPU fallback: every call that computes goes to the CUDA library,
and loading fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from . import abi
from .abi import (RestirBvhDesc, RestirDiReservoirs, RestirFrameInput, RestirFramePlan, RestirFrameState,
                  RestirGBuffer, RestirGiHistory, RestirGiReservoirs, RestirLightsDesc, RestirMeshDesc,
                  RestirParams, RestirScene, RestirSettings, RestirDisplayParams)

# RESTIR_LIBRARY selects another build of the same library (tuning variants).
LIBRARY_PATH = Path(os.environ.get("RESTIR_LIBRARY", Path(__file__).resolve().parent / "librestir_gpu.so"))

SCENE_CORNELL, SCENE_COURTYARD, SCENE_CITY, SCENE_CITY_LIT = 0, 1, 2, 3
GRID_ATOMIC, GRID_DETERMINISTIC = 0, 1
RAY_SCREEN, RAY_HYBRID, RAY_BVH = 0, 1, 2
# restir_gpu.h status codes
OK, ERROR_INVALID_ARGUMENT, ERROR_LAUNCH, ERROR_STEP_CAP, ERROR_UNSUPPORTED = 0, -1, -2, -3, -4
ERROR_TIMEOUT, ERROR_OUT_OF_MEMORY, ERROR_TOO_LARGE = -5, -6, -7
TRACE_CLOSEST, TRACE_ANY, TRACE_CLOSEST_STACKLESS, TRACE_CLOSEST_WATERTIGHT, TRACE_CLOSEST_QUEUE = 0, 1, 2, 3, 4
TRACE_ANY_WAVE = 5
PASS_NAMES = ["shadow", "gbuffer", "di_temporal", "di_spatial", "grid", "gi_temporal", "gi_spatial",
              "denoise", "composite", "reference", "cache", "display", "specular"]

_lib = None

P = C.c_void_p
u32 = C.c_uint32
i32 = C.c_int32

_SIGNATURES = {
    # restir_gpu.h
    "restir_trace": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirScene), P, P, P, u32, C.c_int, P]),
    "restir_shadow_atlas": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirScene), P, P]),
    "restir_gbuffer_primary": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirScene), C.POINTER(RestirGBuffer), P]),
    "restir_grid_clear": (C.c_int, [C.POINTER(RestirParams), P, P]),
    "restir_grid_insert": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirGBuffer), P, P]),
    "restir_di_temporal": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirScene), C.POINTER(RestirGBuffer),
                                     C.POINTER(RestirDiReservoirs), C.POINTER(RestirDiReservoirs), P]),
    "restir_di_spatial": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirScene), C.POINTER(RestirGBuffer),
                                    C.POINTER(RestirDiReservoirs), P, P, P]),
    "restir_gi_temporal": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirScene), C.POINTER(RestirGBuffer),
                                     C.POINTER(RestirGiHistory), P, P, P, C.POINTER(RestirGiReservoirs), P]),
    "restir_gi_temporal_workspace_bytes": (C.c_uint64, [C.POINTER(RestirParams)]),
    "restir_gi_temporal_wavefront": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirScene),
                                               C.POINTER(RestirGBuffer), C.POINTER(RestirGiHistory), P, P, P,
                                               C.POINTER(RestirGiReservoirs), P, C.c_uint64, P]),
    "restir_gi_spatial": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirScene), C.POINTER(RestirGBuffer),
                                    C.POINTER(RestirGiReservoirs), P, C.POINTER(RestirGiHistory), P, P, P, P, P]),
    "restir_svgf_variance": (C.c_int, [C.POINTER(RestirParams), P, P, P, P, P, P]),
    "restir_svgf_atrous": (C.c_int, [C.POINTER(RestirParams), C.c_int, P, P, P, P, P]),
    "restir_composite": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirGBuffer), P, P, P, P, P, P]),
    "restir_composite_specular": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirGBuffer), P, P, P, P, P, P, P]),
    "restir_gi_from_cache": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirScene), C.POINTER(RestirGBuffer), P, P, P,
                                       C.c_uint64, C.POINTER(RestirGiReservoirs), P, P, P]),
    "restir_gi_specular": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirScene), C.POINTER(RestirGBuffer),
                                     C.POINTER(RestirGiHistory), P, P, P, P, P, P]),
    "restir_gi_specular_workspace_bytes": (C.c_uint64, [C.POINTER(RestirParams)]),
    "restir_gi_specular_wavefront": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirScene),
                                               C.POINTER(RestirGBuffer), C.POINTER(RestirGiHistory), P, P, P, P, P,
                                               P, C.c_uint64, P]),
    "restir_reference_accumulate": (C.c_int, [C.POINTER(RestirParams), P, P, P, u32, P]),
    "restir_error_scratch_bytes": (C.c_uint64, [u32, u32]),
    "restir_error": (C.c_int, [C.POINTER(RestirParams), P, P, P, P, P, P]),
    "restir_error_noalloc": (C.c_int, [C.POINTER(RestirParams), P, P, P, P, P]),
    # restir_display.h
    "restir_display_params": (C.c_int, [P, P, u32, u32, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                        C.c_float, C.c_int, C.c_int, C.c_int, C.POINTER(RestirDisplayParams)]),
    "restir_exposure": (C.c_int, [C.POINTER(RestirDisplayParams), P, P, P]),
    "restir_taa": (C.c_int, [C.POINTER(RestirDisplayParams), P, P, P, P, P]),
    "restir_tonemap": (C.c_int, [C.POINTER(RestirDisplayParams), P, P, P, P, P, P]),
    "restir_display": (C.c_int, [C.POINTER(RestirDisplayParams), P, P, P, P, P, P, P, P, P]),
    "restir_struct_size": (C.c_uint64, [C.c_char_p]),
    "restir_status": (C.c_int, [C.POINTER(u32)]),
    "restir_numeric_eval": (C.c_int, [C.c_int, P, P, u32, P]),
    "restir_counters": (C.c_int, [C.c_int, P]),
    "restir_gather_probe": (C.c_int, [P, u32, u32, u32, u32, P, P]),
    "restir_renderer_profile_frame": (C.c_int, [P, C.POINTER(RestirFrameInput), P]),
    "restir_renderer_pass_history": (C.c_int, [P, u32, P]),
    # restir_host.h
    "restir_bvh_build_gpu": (P, [C.POINTER(RestirMeshDesc), P]),
    "restir_mesh_procedural": (P, [C.c_int, u32, u32]),
    "restir_mesh_create": (P, [C.POINTER(RestirMeshDesc)]),
    "restir_mesh_load_gltf": (P, [C.c_char_p, C.c_char_p, u32]),
    "restir_mesh_describe": (C.c_int, [P, C.POINTER(RestirMeshDesc)]),
    "restir_mesh_destroy": (None, [P]),
    "restir_bvh_build": (P, [C.POINTER(RestirMeshDesc), C.c_int]),
    "restir_bvh_describe": (C.c_int, [P, C.POINTER(RestirBvhDesc)]),
    "restir_bvh_destroy": (None, [P]),
    "restir_lights_build": (P, [P, C.c_int, C.c_int, C.c_float, u32, P, P, C.c_float]),
    "restir_lights_describe": (C.c_int, [P, C.POINTER(RestirLightsDesc)]),
    "restir_lights_destroy": (None, [P]),
    "restir_camera_matrices": (None, [P, C.c_float, C.c_float, C.c_float, P, C.c_float, P, P]),
    # restir_frame.h
    "restir_settings_default": (None, [C.POINTER(RestirSettings)]),
    "restir_frame_params": (C.c_int, [C.POINTER(RestirSettings), C.POINTER(RestirMeshDesc), u32,
                                      C.POINTER(RestirBvhDesc), C.POINTER(RestirFrameInput),
                                      C.POINTER(RestirFrameState), C.POINTER(RestirParams),
                                      C.POINTER(RestirFramePlan)]),
    "restir_frame_advance": (None, [C.POINTER(RestirParams), C.POINTER(RestirFramePlan), C.POINTER(RestirFrameInput),
                                    C.POINTER(RestirFrameState)]),
    "restir_renderer_create": (P, [C.POINTER(RestirSettings)]),
    "restir_renderer_destroy": (None, [P]),
    "restir_renderer_set_scene": (C.c_int, [P, P, C.c_int]),
    "restir_renderer_set_settings": (C.c_int, [P, C.POINTER(RestirSettings)]),
    "restir_renderer_get_settings": (C.c_int, [P, C.POINTER(RestirSettings)]),
    "restir_renderer_render": (C.c_int, [P, C.POINTER(RestirFrameInput)]),
    "restir_renderer_render_graph": (C.c_int, [P, C.POINTER(RestirFrameInput)]),
    "restir_renderer_measure": (C.c_int, [P, C.POINTER(abi.RestirMetrics)]),
    "restir_renderer_set_reference_accumulation": (None, [P, C.c_int]),
    "restir_renderer_invalidate_history": (None, [P]),
    "restir_renderer_synchronize": (C.c_int, [P]),
    "restir_renderer_stream": (P, [P]),
    "restir_renderer_last_frame": (C.c_int, [P, C.POINTER(RestirParams), C.POINTER(RestirFramePlan),
                                             C.POINTER(RestirFrameState)]),
    "restir_renderer_buffer": (C.c_int, [P, C.c_char_p, C.POINTER(P), C.POINTER(C.c_uint64)]),
    "restir_renderer_save_state": (C.c_int, [P, C.c_char_p]),
    "restir_renderer_load_state": (C.c_int, [P, C.c_char_p]),
    "restir_batch_create": (P, [C.POINTER(RestirSettings), u32]),
    "restir_batch_destroy": (None, [P]),
    "restir_batch_set_scene": (C.c_int, [P, P, C.c_int]),
    "restir_batch_set_settings": (C.c_int, [P, C.POINTER(RestirSettings)]),
    "restir_batch_render": (C.c_int, [P, C.POINTER(RestirFrameInput)]),
    "restir_batch_autotune": (C.c_int, [P, C.POINTER(RestirFrameInput), u32, C.POINTER(abi.RestirBatchTuning)]),
    "restir_batch_set_tuning": (C.c_int, [P, C.POINTER(abi.RestirBatchTuning)]),
    "restir_batch_get_tuning": (C.c_int, [P, C.POINTER(abi.RestirBatchTuning)]),
    "restir_batch_synchronize": (C.c_int, [P]),
    "restir_batch_stream": (P, [P]),
    "restir_batch_view_buffer": (C.c_int, [P, u32, C.c_char_p, C.POINTER(P), C.POINTER(C.c_uint64)]),
    "restir_batch_view_last_frame": (C.c_int, [P, u32, C.POINTER(RestirParams), C.POINTER(RestirFramePlan),
                                               C.POINTER(RestirFrameState)]),
    "restir_ray_queue_bytes": (C.c_uint64, [u32]),
    "restir_ray_queue_reset": (C.c_int, [P, P]),
    "restir_gi_candidate_records_bytes": (C.c_uint64, [C.POINTER(RestirParams)]),
    "restir_gi_temporal_candidates": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirScene), C.POINTER(RestirGBuffer),
                                                C.POINTER(RestirGiHistory), P, P, P, P, C.c_uint64, P, u32, P]),
    "restir_trace_queue": (C.c_int, [C.POINTER(RestirScene), P, u32, u32, u32, P]),
    "restir_gi_temporal_shade": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirScene), C.POINTER(RestirGBuffer),
                                           C.POINTER(RestirGiHistory), P, P, P, C.POINTER(RestirGiReservoirs), P,
                                           C.c_uint64, P, u32, P]),
    # restir_cache.h
    "restir_cache_config_default": (None, [C.POINTER(abi.RestirCacheConfig)]),
    "restir_cache_layout": (C.c_int, [C.POINTER(abi.RestirCacheConfig), C.POINTER(abi.RestirCacheLayout)]),
    "restir_cache_state_bytes": (C.c_uint64, [C.POINTER(abi.RestirCacheConfig)]),
    "restir_cache_init": (C.c_int, [C.POINTER(abi.RestirCacheConfig), P, P]),
    "restir_cache_query": (C.c_int, [C.POINTER(abi.RestirCacheConfig), P, P, u32, P, P]),
    "restir_cache_features": (C.c_int, [C.POINTER(abi.RestirCacheConfig), P, P, u32, P, P]),
    "restir_cache_forward": (C.c_int, [C.POINTER(abi.RestirCacheConfig), P, P, u32, P, P]),
    "restir_cache_gradients": (C.c_int, [C.POINTER(abi.RestirCacheConfig), P, P, P, u32, P]),
    "restir_cache_adam": (C.c_int, [C.POINTER(abi.RestirCacheConfig), P, P]),
    "restir_cache_train": (C.c_int, [C.POINTER(abi.RestirCacheConfig), P, P, P, u32, P]),
    "restir_gi_temporal_cached": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirScene), C.POINTER(RestirGBuffer),
                                            C.POINTER(RestirGiHistory), P, P, P, C.POINTER(RestirGiReservoirs),
                                            C.POINTER(abi.RestirCacheConfig), P, P, C.c_uint64, P]),
    "restir_gi_spatial_cached": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirScene), C.POINTER(RestirGBuffer),
                                           C.POINTER(RestirGiReservoirs), P, C.POINTER(RestirGiHistory), P, P, P, P,
                                           C.POINTER(abi.RestirCacheConfig), P, P, C.c_uint64, P]),
    "restir_cache_wait_check": (C.c_int, [u32, P, P]),
    "restir_cache_train_frame": (C.c_int, [C.POINTER(RestirParams), C.POINTER(RestirScene), C.POINTER(RestirGBuffer),
                                           P, C.POINTER(abi.RestirCacheConfig), P, P, C.c_uint64, P]),
}


def load() -> C.CDLL:
    """The CUDA library. Raises if it has not been built (python -m restir_b200.build)."""
    global _lib
    if _lib is None:
        if not LIBRARY_PATH.exists():
            raise RuntimeError(f"{LIBRARY_PATH} is missing: build it with `python -m restir_b200.build`")
        lib = C.CDLL(str(LIBRARY_PATH))
        for name, (restype, argtypes) in _SIGNATURES.items():
            if not hasattr(lib, name):
                raise RuntimeError(f"{LIBRARY_PATH} does not export {name}")
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
    return _lib


def ptr(x) -> int | None:
    """Address of a torch tensor, numpy array, ctypes object or int (None for None)."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    return C.addressof(x)


def check(status: int, what: str) -> None:
    if status != 0:
        raise RuntimeError(f"{what} failed with status {status}")


# --- host scene preparation ------------------------------------------------------------------------


class Mesh:
    """A triangle soup (restir_host.h): procedural or from arrays."""

    def __init__(self, handle: int):
        if not handle:
            raise RuntimeError("mesh creation failed")
        self.handle = handle
        self.desc = RestirMeshDesc()
        check(load().restir_mesh_describe(handle, C.byref(self.desc)), "restir_mesh_describe")

    @classmethod
    def procedural(cls, kind: int, seed: int = 0, triangles: int = 0) -> "Mesh":
        return cls(load().restir_mesh_procedural(kind, seed, triangles))

    @classmethod
    def load_gltf(cls, path) -> "Mesh":
        """A mesh from a .gltf or .glb file (restir_mesh_load_gltf)."""
        error = C.create_string_buffer(512)
        handle = load().restir_mesh_load_gltf(str(path).encode(), error, len(error))
        if not handle:
            raise RuntimeError(f"restir_mesh_load_gltf: {error.value.decode(errors='replace')}")
        return cls(handle)

    @classmethod
    def from_arrays(cls, positions: np.ndarray, triangle_material: np.ndarray, materials: np.ndarray,
                    normals: np.ndarray | None = None) -> "Mesh":
        """A mesh from host arrays (copied): 9 floats per triangle, a material index per
        triangle, 8 floats per material (base rgb, roughness, emission rgb, metallic);
        normals (3 per triangle) default to the geometric ones."""
        positions = np.ascontiguousarray(positions, np.float32).reshape(-1)
        triangle_material = np.ascontiguousarray(triangle_material, np.uint32).reshape(-1)
        materials = np.ascontiguousarray(materials, np.float32).reshape(-1)
        d = RestirMeshDesc()
        d.triangle_count = len(triangle_material)
        d.positions = positions.ctypes.data
        if normals is not None:
            normals = np.ascontiguousarray(normals, np.float32).reshape(-1)
            d.normals = normals.ctypes.data
        d.triangle_material = triangle_material.ctypes.data
        d.material_count = len(materials) // 8
        d.materials = materials.ctypes.data
        return cls(load().restir_mesh_create(C.byref(d)))

    @property
    def triangle_count(self) -> int:
        return self.desc.triangle_count

    def positions(self) -> np.ndarray:
        return np.ctypeslib.as_array(C.cast(self.desc.positions, C.POINTER(C.c_float)),
                                     (self.triangle_count * 9,)).copy()

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.restir_mesh_destroy(self.handle)
            self.handle = None


class Bvh:
    """The reference layout (src/bvh.h) built by this library's host builder,
    or on the GPU (device=True: restir_bvh_build_gpu, the same buffer)."""

    def __init__(self, mesh: Mesh, threads: int = 0, device: bool = False):
        if device:
            self.handle = load().restir_bvh_build_gpu(C.byref(mesh.desc), None)
        else:
            threads = threads or (os.cpu_count() or 1)
            self.handle = load().restir_bvh_build(C.byref(mesh.desc), threads)
        if not self.handle:
            raise RuntimeError("restir_bvh_build_gpu failed" if device else "restir_bvh_build failed")
        self.desc = RestirBvhDesc()
        check(load().restir_bvh_describe(self.handle, C.byref(self.desc)), "restir_bvh_describe")
        d = self.desc
        fp = C.POINTER(C.c_float)
        self.data = np.ctypeslib.as_array(C.cast(d.data, fp), (d.float_count,)).copy()
        n = d.triangle_count
        self.triangle_normals = np.ctypeslib.as_array(C.cast(d.triangle_normals, fp), (n * 4,)).copy() if n else \
            np.zeros(0, np.float32)
        self.order = np.ctypeslib.as_array(C.cast(d.order, C.POINTER(C.c_uint32)), (n,)).copy() if n else \
            np.zeros(0, np.uint32)

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.restir_bvh_destroy(self.handle)
            self.handle = None


class Lights:
    """The DI light list (src/lights.h layout)."""

    def __init__(self, bvh: Bvh, mesh: Mesh, settings: RestirSettings, include_emitters: bool = True):
        radius = mesh.desc.radius
        scale = (radius / 1.75) ** 2
        lo = (C.c_float * 3)(*mesh.desc.bounds_min)
        hi = (C.c_float * 3)(*mesh.desc.bounds_max)
        self.handle = load().restir_lights_build(bvh.handle, int(include_emitters and settings.emissive_lighting),
                                                 settings.extra_lights, settings.extra_intensity,
                                                 settings.extra_seed, lo, hi, scale)
        desc = RestirLightsDesc()
        check(load().restir_lights_describe(self.handle, C.byref(desc)), "restir_lights_describe")
        self.count = desc.count
        self.triangles = desc.triangles
        self.data = np.ctypeslib.as_array(C.cast(desc.data, C.POINTER(C.c_float)), (desc.count * 16,)).copy() \
            if desc.count else np.zeros(16, np.float32)

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.restir_lights_destroy(self.handle)
            self.handle = None


def default_settings(mesh: Mesh | None = None) -> RestirSettings:
    """Settings defaults (settings.h:183-227), with the scene's light and sky when given (main.cpp:539-565)."""
    s = RestirSettings()
    load().restir_settings_default(C.byref(s))
    if mesh is not None:
        for k in range(3):
            s.light_position[k] = mesh.desc.light_position[k]
        s.sky_enabled = mesh.desc.sky
    return s


def frame_params(settings: RestirSettings, mesh: Mesh, light_count: int, bvh: Bvh, frame_input: RestirFrameInput,
                 state: RestirFrameState) -> tuple[RestirParams, RestirFramePlan]:
    params = RestirParams()
    plan = RestirFramePlan()
    check(load().restir_frame_params(C.byref(settings), C.byref(mesh.desc), light_count, C.byref(bvh.desc),
                                     C.byref(frame_input), C.byref(state), C.byref(params), C.byref(plan)),
          "restir_frame_params")
    return params, plan


def initial_state() -> RestirFrameState:
    state = RestirFrameState()
    for i in range(4):
        state.previous_view_proj[i * 5] = 1.0
        state.previous_unjittered_view_proj[i * 5] = 1.0
    return state


def frame_input(mesh: Mesh, width: int, height: int, eye=None, yaw=None, pitch=None,
                delta_time: float = 1.0 / 60.0) -> RestirFrameInput:
    fi = RestirFrameInput()
    fi.width, fi.height = width, height
    fi.delta_time = delta_time
    e = eye if eye is not None else mesh.desc.camera_eye
    for k in range(3):
        fi.eye[k] = e[k]
    fi.yaw = mesh.desc.camera_yaw if yaw is None else yaw
    fi.pitch = mesh.desc.camera_pitch if pitch is None else pitch
    return fi


def advance(params: RestirParams, plan: RestirFramePlan, frame_input: RestirFrameInput, state: RestirFrameState):
    load().restir_frame_advance(C.byref(params), C.byref(plan), C.byref(frame_input), C.byref(state))


class Renderer:
    """The reference's Renderer (src/renderer.h:73-125) over the C++ frame driver.

    init(settings) / set_scene(mesh) / render(frame_input) / invalidate_history() /
    set_reference_accumulation(on) / frame_submitted() -> metrics, as in the reference;
    render_graph() replays the frame as one CUDA graph. Work is enqueued on the
    renderer's own CUDA stream; frame_submitted() waits for it.
    """

    def __init__(self, settings: RestirSettings | None = None):
        lib = load()
        self._lib = lib
        self.handle = lib.restir_renderer_create(C.byref(settings) if settings is not None else None)
        if not self.handle:
            raise RuntimeError("restir_renderer_create failed")
        self.mesh = None

    def set_scene(self, mesh: Mesh, use_scene_defaults: bool = True) -> None:
        self.mesh = mesh
        check(self._lib.restir_renderer_set_scene(self.handle, mesh.handle, int(use_scene_defaults)), "set_scene")

    @property
    def settings(self) -> RestirSettings:
        s = RestirSettings()
        check(self._lib.restir_renderer_get_settings(self.handle, C.byref(s)), "get_settings")
        return s

    @settings.setter
    def settings(self, s: RestirSettings) -> None:
        check(self._lib.restir_renderer_set_settings(self.handle, C.byref(s)), "set_settings")

    def render(self, frame_input: RestirFrameInput, graph: bool = False) -> None:
        fn = self._lib.restir_renderer_render_graph if graph else self._lib.restir_renderer_render
        check(fn(self.handle, C.byref(frame_input)), "render")

    def invalidate_history(self) -> None:
        self._lib.restir_renderer_invalidate_history(self.handle)

    def set_reference_accumulation(self, accumulate: bool) -> None:
        self._lib.restir_renderer_set_reference_accumulation(self.handle, int(accumulate))

    def frame_submitted(self) -> abi.RestirMetrics:
        """Error against the reference (cs_error.sc) and per-pass times of the last frame."""
        m = abi.RestirMetrics()
        check(self._lib.restir_renderer_measure(self.handle, C.byref(m)), "measure")
        return m

    def synchronize(self) -> None:
        check(self._lib.restir_renderer_synchronize(self.handle), "synchronize")

    def pass_history(self, frames: int) -> np.ndarray:
        """Per-pass device times (ms) of the last `frames` stream-launched frames: (frames, passes)."""
        ms = np.zeros((frames, len(PASS_NAMES)), np.float32)
        n = self._lib.restir_renderer_pass_history(self.handle, frames, ms.ctypes.data)
        if n < 0:
            raise RuntimeError(f"pass_history failed with status {n}")
        return ms[:n]

    def profile_frame(self, frame_input: RestirFrameInput) -> np.ndarray:
        """One frame with the device work counters on: (passes, 8) counts (see restir_counters)."""
        counts = np.zeros((len(PASS_NAMES), 8), np.uint64)
        check(self._lib.restir_renderer_profile_frame(self.handle, C.byref(frame_input), counts.ctypes.data),
              "profile_frame")
        return counts

    @property
    def stream(self) -> int:
        return self._lib.restir_renderer_stream(self.handle)

    def last_frame(self):
        params, plan, state = RestirParams(), RestirFramePlan(), RestirFrameState()
        check(self._lib.restir_renderer_last_frame(self.handle, C.byref(params), C.byref(plan), C.byref(state)),
              "last_frame")
        return params, plan, state

    def display_image(self) -> np.ndarray:
        """The last frame's tone-mapped image, (height, width, 4) RGBA bytes."""
        params, _, _ = self.last_frame()
        n = params.width * params.height * 4
        bgra = self.download("display", np.uint8)[:n].reshape(params.height, params.width, 4)
        return bgra[..., [2, 1, 0, 3]].copy()

    def buffer(self, name: str) -> tuple[int, int]:
        pointer, nbytes = C.c_void_p(), C.c_uint64()
        check(self._lib.restir_renderer_buffer(self.handle, name.encode(), C.byref(pointer), C.byref(nbytes)),
              f"buffer {name}")
        return pointer.value or 0, nbytes.value

    def save_state(self, path) -> None:
        """The per-frame state (history, reservoirs, grids, ...) to a file (restir_renderer_save_state)."""
        check(self._lib.restir_renderer_save_state(self.handle, str(path).encode()), "save_state")

    def load_state(self, path) -> None:
        """Back from a save_state file; the renderer must have rendered a frame of the same size."""
        check(self._lib.restir_renderer_load_state(self.handle, str(path).encode()), "load_state")

    def download(self, name: str, dtype) -> np.ndarray:
        """A copy of one of the renderer's device buffers (after synchronize)."""
        import torch
        pointer, nbytes = self.buffer(name)
        self.synchronize()
        data = device_view(pointer, nbytes, torch.uint8).cpu()
        return data.numpy().view(dtype)

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.restir_renderer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        if _lib is not None:
            self.close()


def device_view(pointer: int, nbytes: int, dtype):
    """A torch tensor aliasing device memory owned by the library (no copy)."""
    import torch

    class _View:
        def __init__(self):
            self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (pointer, False),
                                             "version": 3}
    return torch.as_tensor(_View(), device="cuda").view(dtype)


def status_flags() -> int:
    flags = C.c_uint32(0)
    check(load().restir_status(C.byref(flags)), "restir_status")
    return flags.value


def cache_config(**overrides) -> abi.RestirCacheConfig:
    """restir_cache_config_default with the given fields replaced."""
    cfg = abi.RestirCacheConfig()
    load().restir_cache_config_default(C.byref(cfg))
    for key, value in overrides.items():
        if key in ("bounds_min", "bounds_max"):
            getattr(cfg, key)[:] = list(value)
        else:
            setattr(cfg, key, value)
    return cfg


def cache_layout(cfg: abi.RestirCacheConfig) -> abi.RestirCacheLayout:
    layout = abi.RestirCacheLayout()
    check(load().restir_cache_layout(C.byref(cfg), C.byref(layout)), "restir_cache_layout")
    return layout


class RadianceCache:
    """The radiance cache of include/restir_cache.h with its state in one torch
    device buffer; queries and targets are torch float32 tensors on the GPU
    ((n, 16) and (n, 4))."""

    def __init__(self, cfg: abi.RestirCacheConfig | None = None, stream: int | None = None):
        import torch
        self.cfg = cfg or cache_config()
        self.layout = cache_layout(self.cfg)
        self._lib = load()
        self.state = torch.zeros(self.layout.bytes, dtype=torch.uint8, device="cuda")
        assert self.state.data_ptr() % 256 == 0
        self.stream = stream
        check(self._lib.restir_cache_init(C.byref(self.cfg), self.state.data_ptr(), stream), "restir_cache_init")

    def region(self, name: str, dtype, count: int | None = None):
        """A view of one region of the state (see RestirCacheLayout)."""
        import torch
        offset = getattr(self.layout, name)
        itemsize = torch.empty((), dtype=dtype).element_size()
        if count is None:
            ends = sorted(getattr(self.layout, f) for f, _ in abi.RestirCacheLayout._fields_[:14])
            count = (ends[ends.index(offset) + 1] - offset) // itemsize
        return self.state[offset:offset + count * itemsize].view(dtype)

    def query(self, queries, out=None):
        import torch
        n = queries.shape[0]
        out = out if out is not None else torch.empty((n, 4), dtype=torch.float16, device="cuda")
        check(self._lib.restir_cache_query(C.byref(self.cfg), self.state.data_ptr(), queries.data_ptr(), n,
                                           out.data_ptr(), self.stream), "restir_cache_query")
        return out

    def forward(self, queries):
        import torch
        out = torch.empty((queries.shape[0], 16), dtype=torch.float32, device="cuda")
        check(self._lib.restir_cache_forward(C.byref(self.cfg), self.state.data_ptr(), queries.data_ptr(),
                                             queries.shape[0], out.data_ptr(), self.stream), "restir_cache_forward")
        return out

    def features(self, queries):
        import torch
        out = torch.empty((queries.shape[0], 64), dtype=torch.int16, device="cuda")
        check(self._lib.restir_cache_features(C.byref(self.cfg), self.state.data_ptr(), queries.data_ptr(),
                                              queries.shape[0], out.data_ptr(), self.stream), "restir_cache_features")
        return out

    def gradients(self, queries, targets) -> None:
        check(self._lib.restir_cache_gradients(C.byref(self.cfg), self.state.data_ptr(), queries.data_ptr(),
                                               targets.data_ptr(), queries.shape[0], self.stream),
              "restir_cache_gradients")

    def adam(self) -> None:
        check(self._lib.restir_cache_adam(C.byref(self.cfg), self.state.data_ptr(), self.stream), "restir_cache_adam")

    def train(self, queries, targets) -> None:
        check(self._lib.restir_cache_train(C.byref(self.cfg), self.state.data_ptr(), queries.data_ptr(),
                                           targets.data_ptr(), queries.shape[0], self.stream), "restir_cache_train")

    def scalars(self) -> abi.RestirCacheScalars:
        raw = self.state[self.layout.scalars:self.layout.scalars + C.sizeof(abi.RestirCacheScalars)].cpu().numpy()
        return abi.RestirCacheScalars.from_buffer_copy(raw.tobytes())


class Batch:
    """Several views of one scene rendered as one frame (include/restir_frame.h,
    restir_batch_*): one scene upload, one shadow atlas, one GI ray queue
    traced by a single persistent launch, one CUDA graph per frame."""

    def __init__(self, settings: RestirSettings | None, views: int):
        self._lib = load()
        self.views = views
        self.handle = self._lib.restir_batch_create(C.byref(settings) if settings is not None else None, views)
        if not self.handle:
            raise RuntimeError("restir_batch_create failed")

    def set_scene(self, mesh: Mesh, use_scene_defaults: bool = True) -> None:
        self.mesh = mesh
        check(self._lib.restir_batch_set_scene(self.handle, mesh.handle, int(use_scene_defaults)), "batch set_scene")

    def set_settings(self, settings: RestirSettings) -> None:
        check(self._lib.restir_batch_set_settings(self.handle, C.byref(settings)), "batch set_settings")

    @staticmethod
    def _inputs(frame_inputs):
        array = (RestirFrameInput * len(frame_inputs))(*frame_inputs)
        return array

    def render(self, frame_inputs) -> None:
        check(self._lib.restir_batch_render(self.handle, self._inputs(frame_inputs)), "batch render")

    def autotune(self, frame_inputs, frames: int = 5) -> abi.RestirBatchTuning:
        best = abi.RestirBatchTuning()
        check(self._lib.restir_batch_autotune(self.handle, self._inputs(frame_inputs), frames, C.byref(best)),
              "batch autotune")
        return best

    @property
    def tuning(self) -> abi.RestirBatchTuning:
        t = abi.RestirBatchTuning()
        check(self._lib.restir_batch_get_tuning(self.handle, C.byref(t)), "batch tuning")
        return t

    @tuning.setter
    def tuning(self, t: abi.RestirBatchTuning) -> None:
        check(self._lib.restir_batch_set_tuning(self.handle, C.byref(t)), "batch tuning")

    @property
    def stream(self) -> int:
        return self._lib.restir_batch_stream(self.handle)

    def synchronize(self) -> None:
        check(self._lib.restir_batch_synchronize(self.handle), "batch synchronize")

    def download(self, view: int, name: str, dtype) -> np.ndarray:
        import torch
        pointer, nbytes = C.c_void_p(), C.c_uint64()
        check(self._lib.restir_batch_view_buffer(self.handle, view, name.encode(), C.byref(pointer), C.byref(nbytes)),
              f"batch buffer {name}")
        self.synchronize()
        return device_view(pointer.value or 0, nbytes.value, torch.uint8).cpu().numpy().view(dtype)

    def last_frame(self, view: int):
        params, plan, state = RestirParams(), RestirFramePlan(), RestirFrameState()
        check(self._lib.restir_batch_view_last_frame(self.handle, view, C.byref(params), C.byref(plan), C.byref(state)),
              "batch last_frame")
        return params, plan, state

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.restir_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
