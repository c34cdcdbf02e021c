"""The host BVH builder and light list against the reference's own
src/bvh.cpp and src/lights.cpp (compiled unmodified in oracle/_ref), and the
layout invariants of src/bvh.h:7-22."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

import oracle.binding as ob
import restir_b200 as rb
from tests.helpers import make_scene, seeded_rays

GOLDEN = Path(__file__).resolve().parent / "golden"


def check_layout(data, node_count, triangle_offset, triangle_count):
    """Every invariant a traversal relies on: children and skip links in range,
    leaves covering every triangle exactly once, boxes containing children."""
    nodes = data[: node_count * 8].reshape(node_count, 8)
    tris = data[triangle_offset * 4:].reshape(triangle_count, 16)
    covered = np.zeros(triangle_count, np.int32)
    for i in range(node_count):
        lo, hi = nodes[i, 0:3], nodes[i, 4:7]
        a, b = nodes[i, 3], nodes[i, 7]
        assert np.all(lo <= hi)
        if b >= 0:
            first, count = int(a), int(b)
            assert count >= 1 and first + count <= triangle_count
            covered[first:first + count] += 1
            v = tris[first:first + count, [0, 1, 2, 4, 5, 6, 8, 9, 10]].reshape(-1, 3)
            assert np.all(v >= lo) and np.all(v <= hi)
        else:
            right, skip = int(a), int(-b) - 1
            assert i + 1 < right < skip <= node_count
            for child in (i + 1, right):
                assert np.all(nodes[child, 0:3] >= lo) and np.all(nodes[child, 4:7] <= hi)
    assert np.all(covered == 1)


def sah_cost(data, node_count):
    nodes = data[: node_count * 8].reshape(node_count, 8)
    ext = nodes[:, 4:7] - nodes[:, 0:3]
    area = 2.0 * (ext[:, 0] * ext[:, 1] + ext[:, 1] * ext[:, 2] + ext[:, 2] * ext[:, 0])
    leaf = nodes[:, 7] >= 0
    return float((area[~leaf].sum() + (area[leaf] * nodes[leaf, 7]).sum()) / area[0])


def mesh_arrays(mesh):
    tm = np.ctypeslib.as_array(C.cast(mesh.desc.triangle_material, C.POINTER(C.c_uint32)),
                               (mesh.triangle_count,)).copy()
    materials = np.ctypeslib.as_array(C.cast(mesh.desc.materials, C.POINTER(C.c_float)),
                                      (mesh.desc.material_count * 8,)).copy().reshape(-1, 8)
    return mesh.positions(), tm, materials


def test_golden_reference_cornell_layout_matches_own_builder():
    g = np.load(GOLDEN / "reference_cornell.npz")
    nodes, offset, depth = (int(v) for v in g["header"])
    check_layout(g["bvh"], nodes, offset, len(g["triangle_material"]))
    setup = make_scene(rb.SCENE_CORNELL)
    np.testing.assert_array_equal(setup.mesh.positions(), g["positions"])
    check_layout(setup.bvh.data, setup.bvh.desc.node_count, setup.bvh.desc.triangle_offset, setup.mesh.triangle_count)
    # The same split rule and the same partition: the same buffer, bit for bit.
    np.testing.assert_array_equal(setup.bvh.data, g["bvh"])
    assert setup.bvh.desc.depth == depth


@pytest.mark.skipif(not ob.reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("kind,triangles", [(rb.SCENE_CORNELL, 0), (rb.SCENE_COURTYARD, 20000), (rb.SCENE_CITY, 60000)])
def test_own_builder_against_reference_builder(kind, triangles):
    mesh = rb.Mesh.procedural(kind, 0, triangles)
    bvh = rb.Bvh(mesh)
    positions, tm, materials = mesh_arrays(mesh)
    ref, nodes, offset, depth = ob.reference_bvh(positions, tm, materials)
    check_layout(bvh.data, bvh.desc.node_count, bvh.desc.triangle_offset, mesh.triangle_count)
    check_layout(ref, nodes, offset, mesh.triangle_count)
    assert sah_cost(bvh.data, bvh.desc.node_count) <= 1.0001 * sah_cost(ref, nodes)
    # Closest hits agree: the same triangle (through the two triangle orders) at the same distance.
    from tests.helpers import SceneSetup
    setup = make_scene(kind, 0, triangles)
    rays = seeded_rays(setup, 20000, seed=5)
    hits = {}
    for name, data, node_count, tri_offset in (("own", bvh.data, bvh.desc.node_count, bvh.desc.triangle_offset),
                                               ("ref", ref, nodes, offset)):
        scene = rb.RestirScene()
        scene.bvh, scene.node_count, scene.triangle_offset = data.ctypes.data, node_count, tri_offset
        ids = np.zeros(len(rays), np.int32)
        t = np.zeros(len(rays), np.float32)
        ob.load().oracle_trace(None, scene, rays.ctypes.data, ids.ctypes.data, t.ctypes.data, len(rays),
                               rb.TRACE_CLOSEST_WATERTIGHT)
        vertices = data[tri_offset * 4:].reshape(-1, 16)[:, [0, 1, 2, 4, 5, 6, 8, 9, 10]]
        key = np.where(ids[:, None] >= 0, vertices[np.maximum(ids, 0)], -1.0)
        hits[name] = (key, t)
    np.testing.assert_array_equal(hits["own"][1], hits["ref"][1])
    np.testing.assert_array_equal(hits["own"][0], hits["ref"][0])


@pytest.mark.skipif(not ob.reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("kind,triangles,extra", [(rb.SCENE_CORNELL, 0, 16), (rb.SCENE_COURTYARD, 20000, 64)])
def test_light_list_matches_reference(kind, triangles, extra):
    mesh = rb.Mesh.procedural(kind, 0, triangles)
    bvh = rb.Bvh(mesh)
    positions, tm, materials = mesh_arrays(mesh)
    ob.reference_bvh(positions, tm, materials)
    settings = rb.default_settings(mesh)
    settings.extra_lights, settings.extra_seed = extra, 7
    own = rb.Lights(bvh, mesh, settings)
    ref, count, triangles_ref = ob.reference_lights(extra, settings.extra_intensity, 7, mesh.desc.bounds_min,
                                                    mesh.desc.bounds_max, (mesh.desc.radius / 1.75) ** 2)
    assert own.count == count and own.triangles == triangles_ref
    own_rows = own.data.reshape(-1, 16)
    ref_rows = ref.reshape(-1, 16)
    # Triangle lights name BVH slots, which differ between builders when the layouts
    # differ: compare them as sets of rows, point lights in order.
    np.testing.assert_array_equal(own_rows[own.triangles:], ref_rows[triangles_ref:])
    if np.array_equal(bvh.data, ob.reference_bvh(positions, tm, materials)[0]):
        np.testing.assert_array_equal(own_rows, ref_rows)


def test_golden_light_list():
    g = np.load(GOLDEN / "reference_cornell.npz")
    setup = make_scene(rb.SCENE_CORNELL)
    settings = rb.default_settings(setup.mesh)
    settings.extra_lights, settings.extra_seed = 16, 7
    own = rb.Lights(setup.bvh, setup.mesh, settings)
    np.testing.assert_array_equal(own.data, g["lights"])
