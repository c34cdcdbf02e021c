"""The oracle against the reference's own shader code.

oracle/_ref/libref_shaders.so is the reference's shader source (bvh.sh,
hashgrid.sh, restir.sh, di.sh, svgf.sh and the compute and fragment passes
that use them) compiled as C++ by oracle/Makefile through a GLSL shim
(oracle/ref_shim). These tests give it and the oracle restatement the same
inputs and require bit-equal outputs, under the numeric conventions of
include/restir_numeric.h (no FMA contraction, exact floor(log2), the
library's own exp/sin/cos). The CUDA kernels are bit-exact against the
oracle in the -m gpu tests, so this closes the chain kernel = restatement =
reference shader. Skipped where the library was not built (the reference's
sources are needed to build it).
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

import oracle.binding as ob
import restir_b200 as rb
from restir_b200.abi import RestirGBuffer, RestirParams, RestirScene
from tests.helpers import gbuffer_struct, host_gbuffer, make_scene, params_for, seeded_rays

LIBRARY = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "libref_shaders.so"
pytestmark = pytest.mark.skipif(not LIBRARY.exists(), reason="oracle/_ref/libref_shaders.so not built")

_lib = None
P = C.c_void_p


def ref():
    global _lib
    if _lib is None:
        lib = C.CDLL(str(LIBRARY))
        lib.ref_trace.argtypes = [C.POINTER(RestirScene), P, P, P, C.c_uint32, C.c_int]
        lib.ref_grid_keys.argtypes = [P, P, C.c_uint32, P, P, P, C.c_uint32, P, P, P]
        lib.ref_grid_insert.argtypes = [C.POINTER(RestirParams), C.POINTER(RestirGBuffer), P]
        _lib = lib
    return _lib


SCENES = {
    "cornell": (rb.SCENE_CORNELL, 0, 0),
    "courtyard20k": (rb.SCENE_COURTYARD, 1, 20000),
    "city60k": (rb.SCENE_CITY, 3, 60000),
}


@pytest.mark.parametrize("scene", list(SCENES))
@pytest.mark.parametrize("kind", [rb.TRACE_CLOSEST, rb.TRACE_ANY, rb.TRACE_CLOSEST_STACKLESS])
def test_traversal_equals_reference_bvh_sh(scene, kind):
    """Closest-hit ids (shared short stack, bvh.sh:216-295, and stackless
    walk, 140-174) and any-hit ids, with their distances, equal the
    reference's traversal bit for bit on seeded rays (a quarter of them axis
    parallel)."""
    setup = make_scene(*SCENES[scene])
    rays = seeded_rays(setup, 20000, seed=7)
    want_ids = np.zeros(len(rays), np.int32)
    want_t = np.zeros(len(rays), np.float32)
    got_ids, got_t = np.zeros_like(want_ids), np.zeros_like(want_t)
    assert ob.load().oracle_trace(None, setup.host_scene(), rays.ctypes.data, got_ids.ctypes.data,
                                  got_t.ctypes.data, len(rays), kind) == 0
    assert ref().ref_trace(setup.host_scene(), rays.ctypes.data, want_ids.ctypes.data, want_t.ctypes.data,
                           len(rays), kind) == 0
    np.testing.assert_array_equal(got_ids, want_ids)
    np.testing.assert_array_equal(got_t.view(np.uint32), want_t.view(np.uint32))
    assert (want_ids >= 0).mean() > 0.3


def test_grid_keys_equal_reference_hashgrid_sh():
    """gridCellSize, gridJitter and gridKey (hashgrid.sh:82-127): cell size
    bits, first slot and checksum for seeded positions over three orders of
    magnitude of camera distance, axis-aligned and random normals."""
    rng = np.random.default_rng(5)
    n = 50000
    positions = (rng.normal(size=(n, 3)) * np.exp(rng.uniform(-3.0, 4.0, (n, 1)))).astype(np.float32)
    normals = rng.normal(size=(n, 3))
    normals[: n // 4] = np.eye(3)[rng.integers(0, 3, n // 4)] * rng.choice([-1.0, 1.0], (n // 4, 1))
    normals = (normals / np.linalg.norm(normals, axis=1, keepdims=True)).astype(np.float32)
    randoms = rng.random((n, 2), dtype=np.float32)
    camera = np.array([0.3, 1.2, -2.5], np.float32)
    constants = np.array([0.02, 0.0021, 6.0], np.float32)
    outputs = {side: [np.zeros(n, np.uint32) for _ in range(3)] for side in ("oracle", "ref")}
    args = (camera.ctypes.data, constants.ctypes.data, 65536, positions.ctypes.data, normals.ctypes.data,
            randoms.ctypes.data, n)
    ob.load().oracle_grid_keys(*args, *(a.ctypes.data for a in outputs["oracle"]))
    assert ref().ref_grid_keys(*args, *(a.ctypes.data for a in outputs["ref"])) == 0
    for got, want, name in zip(outputs["oracle"], outputs["ref"], ("cell size", "slot", "checksum")):
        np.testing.assert_array_equal(got, want, err_msg=name)
    assert len(np.unique(outputs["ref"][0])) >= 6  # many cell sizes


@pytest.mark.parametrize("scene,size", [("cornell", (96, 96)), ("courtyard20k", (160, 90))])
def test_grid_insert_equals_reference_cs_grid_insert(scene, size):
    """The whole grid after cs_grid_insert.sc (checksums, counts and entries)
    equals the oracle's deterministic-mode grid on a G-buffer rendered by the
    oracle: the reference's invocations run in pixel order, where its first
    32 arrivals are the lowest pixel indices."""
    setup = make_scene(*SCENES[scene])
    w, h = size
    params, _ = params_for(setup, w, h, gi_divisor=1 if scene == "cornell" else 2)
    params.grid_mode = rb.GRID_DETERMINISTIC
    gbuffer = host_gbuffer(w, h)
    ob.load().oracle_gbuffer_primary(params, setup.host_scene(), gbuffer_struct(gbuffer))
    T, cap = params.grid_table_size, params.grid_cell_capacity
    assert (T, cap) == (65536, 32)
    got = np.zeros(T * (2 + cap), np.uint32)
    want = np.zeros_like(got)
    ob.load().oracle_grid_insert(params, gbuffer_struct(gbuffer), got.ctypes.data)
    assert ref().ref_grid_insert(params, gbuffer_struct(gbuffer), want.ctypes.data) == 0
    np.testing.assert_array_equal(got, want)
    assert np.count_nonzero(want[:T]) > 20


FRAME_CASES = {
    # Cornell box, full-resolution GI, point light and emissive panel.
    "cornell": dict(scene=(rb.SCENE_CORNELL, 0, 0), size=(64, 64), frames=3, overrides=dict(gi_divisor=1)),
    # Courtyard with sky, half-resolution GI, 64 extra point lights and the emissive triangles in DI.
    "courtyard": dict(scene=(rb.SCENE_COURTYARD, 0, 20000), size=(128, 72), frames=3,
                      overrides=dict(extra_lights=64)),
    # Every GI ray through the BVH, 4 candidates per pixel.
    "bvh-rays": dict(scene=(rb.SCENE_CORNELL, 0, 0), size=(48, 48), frames=2,
                     overrides=dict(gi_divisor=1, ray_mode=rb.RAY_BVH, initial_candidates=4)),
    # Depth buffer only, screen-space reuse, GI without DI, no denoiser.
    "screen-space": dict(scene=(rb.SCENE_COURTYARD, 0, 20000), size=(96, 54), frames=3,
                         overrides=dict(ray_mode=rb.RAY_SCREEN, world_space_reuse=0, direct_lighting=1,
                                        denoiser=0)),
}


@pytest.mark.parametrize("case", list(FRAME_CASES))
def test_frame_passes_equal_reference_shaders(case):
    """Every pass the reference runs as a compute or fragment shader (grid
    insert, GI temporal with its 4x8 groups and barriers, GI spatial, DI
    temporal and spatial, SVGF variance and a-trous, composite, specular),
    over frames that carry history, gives the oracle's outputs bit for bit
    when both get the same inputs."""
    from oracle.frame import run_pinned
    c = FRAME_CASES[case]
    setup = make_scene(*c["scene"], extra_lights=c["overrides"].get("extra_lights", 0))
    settings = setup.settings
    for k, v in c["overrides"].items():
        setattr(settings, k, v)
    settings.grid_mode = rb.GRID_DETERMINISTIC
    if "extra_lights" in c["overrides"]:
        setup.lights = rb.Lights(setup.bvh, setup.mesh, settings)
    w, h = c["size"]
    report, pinned = run_pinned(setup, w, h, c["frames"], settings)
    assert report == {}, report
    expected = {"grid_insert", "gi_temporal", "gi_spatial", "composite_specular"}
    if case != "screen-space":
        expected |= {"di_temporal", "di_spatial", "svgf_variance", "svgf_atrous", "gi_specular"}
    assert expected <= set(pinned), pinned
    # Every pinned pass wrote output, so the equality is not of untouched buffers.
    assert all(pinned[name] > 0 for name in expected), pinned
