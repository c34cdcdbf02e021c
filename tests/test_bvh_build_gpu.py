"""The device BVH builder (restir_bvh_build_gpu) against the host builder
(itself bit-identical to the reference's bvh.cpp on the Cornell box, see
test_bvh_layout.py): the same buffer bit for bit (nodes, skip links, leaf
ranges, triangle records), the same BVH-slot order, shading normals and
emitters, on procedural scenes of every size class, random triangle soups,
coincident centroids (the median split) and the smallest inputs."""
import ctypes as C

import numpy as np
import pytest

import restir_b200 as rb

pytestmark = pytest.mark.gpu


def emitters(bvh):
    d = bvh.desc
    if d.emitter_count == 0:
        return np.zeros(0, np.float32)
    return np.ctypeslib.as_array(C.cast(d.emitters, C.POINTER(C.c_float)), (d.emitter_count * 13,)).copy()


def assert_same(mesh):
    host = rb.Bvh(mesh)
    device = rb.Bvh(mesh, device=True)
    assert device.desc.node_count == host.desc.node_count
    assert device.desc.triangle_offset == host.desc.triangle_offset
    assert device.desc.depth == host.desc.depth
    np.testing.assert_array_equal(device.order, host.order)
    np.testing.assert_array_equal(device.data.view(np.uint32), host.data.view(np.uint32))
    np.testing.assert_array_equal(device.triangle_normals.view(np.uint32), host.triangle_normals.view(np.uint32))
    np.testing.assert_array_equal(emitters(device), emitters(host))
    return host, device


@pytest.mark.parametrize("kind,triangles", [(rb.SCENE_CORNELL, 0), (rb.SCENE_COURTYARD, 20000),
                                            (rb.SCENE_COURTYARD, 100000), (rb.SCENE_CITY, 300000)])
def test_device_builder_equals_host_builder(kind, triangles):
    mesh = rb.Mesh.procedural(kind, 3, triangles)
    host, _ = assert_same(mesh)
    assert host.desc.node_count > 1


def soup(n, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-10.0, 10.0, (n, 1, 3))
    positions = (centres + rng.normal(0.0, scale, (n, 3, 3))).astype(np.float32)
    materials = np.array([[0.7, 0.6, 0.5, 0.8, 0.0, 0.0, 0.0, 0.1],
                          [0.2, 0.3, 0.4, 0.5, 4.0, 3.0, 2.0, 0.0]], np.float32)
    return positions, (rng.random(n) < 0.05).astype(np.uint32), materials


@pytest.mark.parametrize("n,seed", [(1, 0), (2, 1), (65, 2), (4097, 3), (50000, 4)])
def test_device_builder_on_random_soups(n, seed):
    positions, tm, materials = soup(n, seed)
    assert_same(rb.Mesh.from_arrays(positions, tm, materials))


def test_device_builder_median_split_of_coincident_centroids():
    # 3000 triangles in 30 stacks of 100 copies with the same centroid and
    # different extents: nodes with one centroid and more than 16 triangles
    # are split at their median.
    rng = np.random.default_rng(9)
    stacks = rng.integers(-20, 20, (30, 3)) / 4.0
    positions = []
    for c in stacks:
        for k in range(100):
            # bounds c -+ (a, b, e), all dyadic: the centroid is exactly c in float32
            a, b, e = (k + 1) / 64.0, (k % 7 + 1) / 32.0, (k % 5 + 1) / 16.0
            positions.append([[c[0] + a, c[1] + b, c[2]], [c[0] - a, c[1] - b, c[2] + e], [c[0], c[1], c[2] - e]])
    positions = np.array(positions, np.float32)
    tm = np.zeros(len(positions), np.uint32)
    materials = np.array([[0.5, 0.5, 0.5, 1.0, 0.0, 0.0, 0.0, 0.0]], np.float32)
    host, _ = assert_same(rb.Mesh.from_arrays(positions, tm, materials))
    assert host.desc.depth > 8


def test_renderer_builds_on_the_device():
    setup_mesh = rb.Mesh.procedural(rb.SCENE_COURTYARD, 1, 30000)
    frames = {}
    for on_device in (0, 1):
        settings = rb.default_settings(setup_mesh)
        settings.bvh_on_device = on_device
        settings.grid_mode = rb.GRID_DETERMINISTIC
        renderer = rb.Renderer(settings)
        renderer.set_scene(setup_mesh, use_scene_defaults=False)
        frame = rb.frame_input(setup_mesh, 96, 64)
        for _ in range(2):
            renderer.render(frame)
        frames[on_device] = (renderer.download("bvh", np.uint32), renderer.download("display.hdr", np.uint16))
    np.testing.assert_array_equal(frames[0][0], frames[1][0])
    np.testing.assert_array_equal(frames[0][1], frames[1][1])
