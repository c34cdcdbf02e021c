"""ORACLE (test infrastructure): ctypes binding of oracle/liboracle.so, of
the reference's own BVH and light-list builders compiled in oracle/_ref, and
of the reference's own shader code compiled there (libref_shaders.so).

The oracle's entry points take the arguments of the CUDA ABI's passes with
host (numpy) buffers instead of device pointers.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

from restir_b200.abi import (RestirDiReservoirs, RestirDisplayParams, RestirGBuffer, RestirGiHistory,
                             RestirGiReservoirs, RestirParams, RestirScene)

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "liboracle.so"
REFERENCE_LIBRARY = HERE / "_ref" / "libref_bvh.so"
SHADER_LIBRARY = HERE / "_ref" / "libref_shaders.so"

P = C.c_void_p
u32 = C.c_uint32
PP = C.POINTER(RestirParams)
PS = C.POINTER(RestirScene)
PG = C.POINTER(RestirGBuffer)

_SIGNATURES = {
    "oracle_trace": (C.c_int, [PP, PS, P, P, P, u32, C.c_int]),
    "oracle_shadow_atlas": (C.c_int, [PP, PS, P]),
    "oracle_gbuffer_primary": (C.c_int, [PP, PS, PG]),
    "oracle_grid_clear": (C.c_int, [PP, P]),
    "oracle_grid_insert": (C.c_int, [PP, PG, P]),
    "oracle_di_temporal": (C.c_int, [PP, PS, PG, C.POINTER(RestirDiReservoirs), C.POINTER(RestirDiReservoirs)]),
    "oracle_di_spatial": (C.c_int, [PP, PS, PG, C.POINTER(RestirDiReservoirs), P, P]),
    "oracle_gi_temporal": (C.c_int, [PP, PS, PG, C.POINTER(RestirGiHistory), P, P, P, C.POINTER(RestirGiReservoirs)]),
    "oracle_gi_spatial": (C.c_int, [PP, PS, PG, C.POINTER(RestirGiReservoirs), P, C.POINTER(RestirGiHistory), P, P,
                                    P, P]),
    "oracle_gi_temporal_cached": (C.c_int, [PP, PS, PG, C.POINTER(RestirGiHistory), P, P, P,
                                            C.POINTER(RestirGiReservoirs), P]),
    "oracle_gi_spatial_cached": (C.c_int, [PP, PS, PG, C.POINTER(RestirGiReservoirs), P, C.POINTER(RestirGiHistory),
                                           P, P, P, P, P]),
    "oracle_svgf_variance": (C.c_int, [PP, P, P, P, P, P]),
    "oracle_svgf_atrous": (C.c_int, [PP, C.c_int, P, P, P, P]),
    "oracle_composite": (C.c_int, [PP, PG, P, P, P, P, P]),
    "oracle_composite_specular": (C.c_int, [PP, PG, P, P, P, P, P, P]),
    "oracle_gi_specular": (C.c_int, [PP, PS, PG, C.POINTER(RestirGiHistory), P, P, P, P, P]),
    "oracle_reference_accumulate": (C.c_int, [PP, P, P, P, u32]),
    "oracle_error": (C.c_int, [PP, P, P, P, P]),
    "oracle_exposure": (C.c_int, [C.POINTER(RestirDisplayParams), P, P]),
    "oracle_taa": (C.c_int, [C.POINTER(RestirDisplayParams), P, P, P, P]),
    "oracle_tonemap": (C.c_int, [C.POINTER(RestirDisplayParams), P, P, P, P, P]),
    "oracle_last_counts": (None, [P]),
    "oracle_numeric_eval": (None, [C.c_int, P, P, u32]),
    "oracle_grid_keys": (None, [P, P, u32, P, P, P, u32, P, P, P]),
    "oracle_set_threads": (None, [C.c_int]),
    "oracle_get_threads": (C.c_int, []),
    # radiance cache (oracle_cache.cpp): config and layout pointers first
    "oracle_cache_features": (None, [P, P, P, P, u32, P]),
    "oracle_cache_forward": (None, [P, P, u32, P]),
    "oracle_cache_gradients": (None, [P, P, P, P, P, P, u32, C.c_float, P, P, P]),
    "oracle_cache_adam": (None, [P, u32, P, P, P, P, C.c_float, C.c_float]),
}

# The reference's shader passes (oracle/ref_shim/ref_passes.cpp): the
# arguments of the oracle function of the same name.
_SHADER_SIGNATURES = {
    "ref_trace": (C.c_int, [PS, P, P, P, u32, C.c_int]),
    "ref_grid_keys": (C.c_int, [P, P, u32, P, P, P, u32, P, P, P]),
    "ref_grid_insert": (C.c_int, [PP, PG, P]),
    "ref_gi_temporal": _SIGNATURES["oracle_gi_temporal"],
    "ref_gi_spatial": _SIGNATURES["oracle_gi_spatial"],
    "ref_di_temporal": _SIGNATURES["oracle_di_temporal"],
    "ref_di_spatial": _SIGNATURES["oracle_di_spatial"],
    "ref_svgf_variance": _SIGNATURES["oracle_svgf_variance"],
    "ref_svgf_atrous": _SIGNATURES["oracle_svgf_atrous"],
    "ref_composite_specular": _SIGNATURES["oracle_composite_specular"],
    "ref_gi_specular": _SIGNATURES["oracle_gi_specular"],
    "ref_set_threads": (None, [C.c_int]),
    "ref_get_threads": (C.c_int, []),
}

_lib = None
_ref = None
_shaders = None


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            subprocess.run(["make", "-s", "-C", str(HERE), str(LIBRARY)], check=True)
        lib = C.CDLL(str(LIBRARY))
        for name, (restype, argtypes) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
    return _lib


def last_counts() -> dict:
    counts = (C.c_uint64 * 5)()
    load().oracle_last_counts(counts)
    return {"bvh_rays": counts[0], "screen_rays": counts[1], "node_visits": counts[2],
            "triangle_tests": counts[3], "pixels": counts[4]}


def reference_available() -> bool:
    return REFERENCE_LIBRARY.exists()


def load_reference() -> C.CDLL:
    """The reference's src/bvh.cpp + src/lights.cpp, built unmodified by oracle/Makefile."""
    global _ref
    if _ref is None:
        lib = C.CDLL(str(REFERENCE_LIBRARY))
        lib.ref_build_bvh.restype = C.c_uint64
        lib.ref_build_bvh.argtypes = [P, u32, P, P, P, P, u32, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32)]
        lib.ref_copy_bvh.argtypes = [P]
        lib.ref_build_lights.restype = u32
        lib.ref_build_lights.argtypes = [C.c_int, C.c_float, u32, P, P, C.c_float, C.POINTER(u32)]
        lib.ref_copy_lights.argtypes = [P]
        _ref = lib
    return _ref


def reference_bvh(positions: np.ndarray, triangle_material: np.ndarray, materials: np.ndarray):
    """The reference builder's float buffer for a triangle soup. materials: (m, 8) rows
    (base rgb, roughness, emission rgb, metallic)."""
    lib = load_reference()
    positions = np.ascontiguousarray(positions, np.float32)
    tm = np.ascontiguousarray(triangle_material, np.uint32)
    base = np.ascontiguousarray(materials[:, 0:3], np.float32)
    emission = np.ascontiguousarray(materials[:, 4:7], np.float32)
    metallic = np.ascontiguousarray(materials[:, 7], np.float32)
    nodes, offset, depth = u32(), u32(), u32()
    count = lib.ref_build_bvh(positions.ctypes.data, len(tm), tm.ctypes.data, base.ctypes.data, emission.ctypes.data,
                              metallic.ctypes.data, len(materials), C.byref(nodes), C.byref(offset), C.byref(depth))
    data = np.zeros(count, np.float32)
    lib.ref_copy_bvh(data.ctypes.data)
    return data, nodes.value, offset.value, depth.value


def reference_lights(extra_count: int, extra_intensity: float, extra_seed: int, bounds_min, bounds_max,
                     intensity_scale: float):
    """The reference's light list over the last reference_bvh's emitters."""
    lib = load_reference()
    lo = np.asarray(bounds_min, np.float32)
    hi = np.asarray(bounds_max, np.float32)
    triangles = u32()
    count = lib.ref_build_lights(extra_count, extra_intensity, extra_seed, lo.ctypes.data, hi.ctypes.data,
                                 intensity_scale, C.byref(triangles))
    data = np.zeros(count * 16, np.float32)
    if count:
        lib.ref_copy_lights(data.ctypes.data)
    return data, count, triangles.value


def shaders_available() -> bool:
    return SHADER_LIBRARY.exists()


def load_shaders() -> C.CDLL:
    """The reference's shader passes compiled as C++ (oracle/ref_shim), built by oracle/Makefile."""
    global _shaders
    if _shaders is None:
        lib = C.CDLL(str(SHADER_LIBRARY))
        for name, (restype, argtypes) in _SHADER_SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _shaders = lib
    return _shaders
