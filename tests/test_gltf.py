"""The glTF reader (restir_mesh_load_gltf) on files this test writes: a node
hierarchy with a matrix and a translation-rotation-scale child, indexed (8-,
16- and 32-bit) and non-indexed primitives, a primitive without normals and
one without a material, an emissive material with KHR_materials_emissive_strength;
as .gltf with an external buffer, with a data URI, and as .glb. The expected
mesh is computed here with numpy from the glTF 2.0 rules."""
import base64
import ctypes as C
import json
import struct

import numpy as np
import pytest

import restir_b200 as rb


def quat_matrix(q):
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def scene():
    """(gltf dict without buffers, binary blob, expected triangles per material slot)."""
    rng = np.random.default_rng(4)
    blob = bytearray()
    views, accessors = [], []

    def add(array, component, kind):
        nonlocal blob
        while len(blob) % 4:
            blob += b"\0"
        data = np.ascontiguousarray(array).tobytes()
        views.append({"buffer": 0, "byteOffset": len(blob), "byteLength": len(data)})
        count = len(array) if kind == "SCALAR" else len(array) // int(kind[-1])
        accessors.append({"bufferView": len(views) - 1, "componentType": component, "count": count, "type": kind})
        blob += data
        return len(accessors) - 1

    # mesh 0: a 5-vertex fan, 16-bit indices, normals given
    p0 = rng.uniform(-1, 1, (5, 3)).astype(np.float32)
    n0 = rng.normal(size=(5, 3)).astype(np.float32)
    i0 = np.array([0, 1, 2, 0, 2, 3, 0, 3, 4], np.uint16)
    # mesh 1: 6 vertices, no indices, no normals
    p1 = rng.uniform(-2, 2, (6, 3)).astype(np.float32)
    # mesh 2: 8-bit and 32-bit indexed primitives, the second without a material
    p2 = rng.uniform(0, 1, (4, 3)).astype(np.float32)
    n2 = np.tile(np.array([[0, 0, 1]], np.float32), (4, 1))
    i2a = np.array([0, 1, 2], np.uint8)
    i2b = np.array([1, 3, 2, 0, 3, 1], np.uint32)
    a = {"p0": add(p0.reshape(-1), 5126, "VEC3"), "n0": add(n0.reshape(-1), 5126, "VEC3"), "i0": add(i0, 5123, "SCALAR"),
         "p1": add(p1.reshape(-1), 5126, "VEC3"), "p2": add(p2.reshape(-1), 5126, "VEC3"),
         "n2": add(n2.reshape(-1), 5126, "VEC3"), "i2a": add(i2a, 5121, "SCALAR"), "i2b": add(i2b, 5125, "SCALAR")}
    materials = [
        {"pbrMetallicRoughness": {"baseColorFactor": [0.8, 0.2, 0.1, 1.0], "metallicFactor": 0.0, "roughnessFactor": 0.4}},
        {"pbrMetallicRoughness": {"baseColorFactor": [0.9, 0.9, 0.9, 1.0], "metallicFactor": 0.0},
         "emissiveFactor": [1.0, 0.5, 0.25], "extensions": {"KHR_materials_emissive_strength": {"emissiveStrength": 8.0}},
         "doubleSided": True},
        {},  # glTF defaults: white, metallic 1, roughness 1
    ]
    meshes = [
        {"primitives": [{"attributes": {"POSITION": a["p0"], "NORMAL": a["n0"]}, "indices": a["i0"], "material": 2}]},
        {"primitives": [{"attributes": {"POSITION": a["p1"]}, "material": 0}]},
        {"primitives": [{"attributes": {"POSITION": a["p2"], "NORMAL": a["n2"]}, "indices": a["i2a"], "material": 1},
                        {"attributes": {"POSITION": a["p2"], "NORMAL": a["n2"]}, "indices": a["i2b"]}]},
    ]
    root_matrix = np.array([[1, 0, 0, 0.5], [0, 0, -1, 0], [0, 1, 0, 0.25], [0, 0, 0, 1]], np.float64)
    q = np.array([0.0, 0.38268343, 0.0, 0.92387953])
    t, sc = np.array([1.0, -2.0, 0.5]), np.array([2.0, 0.5, 1.5])
    child = np.eye(4)
    child[:3, :3] = quat_matrix(q) @ np.diag(sc)
    child[:3, 3] = t
    nodes = [
        {"matrix": list(root_matrix.T.reshape(-1)), "children": [1, 2]},
        {"mesh": 0},
        {"translation": list(t), "rotation": list(q), "scale": list(sc), "mesh": 1, "children": [3]},
        {"mesh": 2},
    ]
    gltf = {"asset": {"version": "2.0"}, "scene": 0, "scenes": [{"nodes": [0]}], "nodes": nodes, "meshes": meshes,
            "materials": materials, "accessors": accessors, "bufferViews": views}

    def transform(m, p):
        return (np.c_[p.astype(np.float64), np.ones(len(p))] @ m.T)[:, :3]

    world0, world1 = root_matrix, root_matrix @ child
    expected = {0: [], 1: [], 2: [], 3: []}
    expected[2].append(transform(world0, p0)[i0.astype(int)].reshape(-1, 9))
    expected[0].append(transform(world1, p1).reshape(-1, 9))
    expected[1].append(transform(world1, p2)[i2a.astype(int)].reshape(-1, 9))
    expected[3].append(transform(world1, p2)[i2b.astype(int)].reshape(-1, 9))
    return gltf, bytes(blob), {k: np.concatenate(v) for k, v in expected.items()}, (world0, world1, n0, i0, n2)


def write(tmp_path, form):
    gltf, blob, expected, extra = scene()
    if form == "external":
        (tmp_path / "mesh data.bin").write_bytes(blob)
        gltf["buffers"] = [{"byteLength": len(blob), "uri": "mesh%20data.bin"}]
        path = tmp_path / "scene.gltf"
        path.write_text(json.dumps(gltf, indent=1))
    elif form == "data-uri":
        gltf["buffers"] = [{"byteLength": len(blob),
                            "uri": "data:application/octet-stream;base64," + base64.b64encode(blob).decode()}]
        path = tmp_path / "scene.gltf"
        path.write_text(json.dumps(gltf))
    else:
        gltf["buffers"] = [{"byteLength": len(blob)}]
        text = json.dumps(gltf).encode()
        text += b" " * (-len(text) % 4)
        binary = blob + b"\0" * (-len(blob) % 4)
        body = struct.pack("<II", len(text), 0x4E4F534A) + text + struct.pack("<II", len(binary), 0x004E4942) + binary
        path = tmp_path / "scene.glb"
        path.write_bytes(struct.pack("<III", 0x46546C67, 2, 12 + len(body)) + body)
    return path, expected, extra


def mesh_arrays(mesh):
    d = mesh.desc
    n = mesh.triangle_count
    tm = np.ctypeslib.as_array(C.cast(d.triangle_material, C.POINTER(C.c_uint32)), (n,)).copy()
    normals = np.ctypeslib.as_array(C.cast(d.normals, C.POINTER(C.c_float)), (n * 3,)).copy().reshape(n, 3)
    mats = np.ctypeslib.as_array(C.cast(d.materials, C.POINTER(C.c_float)), (d.material_count * 8,)).copy()
    return mesh.positions().reshape(n, 9), tm, normals, mats.reshape(-1, 8)


@pytest.mark.parametrize("form", ["external", "data-uri", "glb"])
def test_gltf_reader(tmp_path, form):
    path, expected, (world0, world1, n0, i0, n2) = write(tmp_path, form)
    mesh = rb.Mesh.load_gltf(path)
    positions, tm, normals, mats = mesh_arrays(mesh)
    # triangles grouped by material slot, in order; the default material last
    want = np.concatenate([expected[k] for k in range(4)])
    np.testing.assert_allclose(positions, want, rtol=0, atol=2e-6)
    np.testing.assert_array_equal(tm, np.repeat(np.arange(4), [len(expected[k]) for k in range(4)]))
    np.testing.assert_allclose(mats[:, :4], [[0.8, 0.2, 0.1, 0.4], [0.9, 0.9, 0.9, 1.0], [1, 1, 1, 1], [1, 1, 1, 1]],
                               atol=1e-7)
    np.testing.assert_allclose(mats[:, 4:7], [[0, 0, 0], [8, 4, 2], [0, 0, 0], [0, 0, 0]])
    np.testing.assert_allclose(mats[:, 7], [0, 0, 1, 1])
    # shading normals: the normalised sum of the corners' world normals
    nt = np.linalg.inv(world0[:3, :3]).T
    corner = (n0.astype(np.float64) @ nt.T)
    corner /= np.linalg.norm(corner, axis=1, keepdims=True)
    s = corner[i0.astype(int)].reshape(-1, 3, 3).sum(axis=1)
    s /= np.linalg.norm(s, axis=1, keepdims=True)
    got = normals[tm == 2]
    np.testing.assert_allclose(got, s, atol=2e-6)
    # no NORMAL: the corners' area-weighted face normals give the face normal of a lone triangle
    tri = positions[tm == 0].reshape(-1, 3, 3).astype(np.float64)
    face = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    face /= np.linalg.norm(face, axis=1, keepdims=True)
    np.testing.assert_allclose(normals[tm == 0], face, atol=1e-5)
    # the light: in front of the emissive triangle's centroid, along its normal, 0.15 radii out
    emit = positions[tm == 1].reshape(3, 3).astype(np.float64)
    nw = np.linalg.inv(world1[:3, :3]).T @ np.array([0, 0, 1.0])
    nw /= np.linalg.norm(nw)
    light = emit.mean(axis=0) + nw * 0.15 * mesh.desc.radius
    np.testing.assert_allclose(list(mesh.desc.light_position), light, atol=1e-5)
    assert mesh.desc.sky == 1
    # the double-sided material reaches the BVH's normal rows (w = 1)
    bvh = rb.Bvh(mesh)
    two_sided = bvh.triangle_normals.reshape(-1, 4)[:, 3]
    np.testing.assert_array_equal(two_sided, (tm[bvh.order] == 1).astype(np.float32))
    assert bvh.desc.emitter_count == 1


def test_gltf_forms_give_the_same_mesh(tmp_path):
    meshes = []
    for form in ("external", "data-uri", "glb"):
        d = tmp_path / form
        d.mkdir()
        path, _, _ = write(d, form)
        meshes.append(mesh_arrays(rb.Mesh.load_gltf(path)))
    for other in meshes[1:]:
        for x, y in zip(meshes[0], other):
            np.testing.assert_array_equal(x, y)


def test_gltf_errors(tmp_path):
    with pytest.raises(RuntimeError, match="cannot open"):
        rb.Mesh.load_gltf(tmp_path / "missing.gltf")
    bad = tmp_path / "bad.gltf"
    bad.write_text("{ \"asset\": ")
    with pytest.raises(RuntimeError, match="JSON"):
        rb.Mesh.load_gltf(bad)
    gltf, blob, _, _ = scene()
    gltf["accessors"][2]["count"] = 10_000  # the 16-bit indices run past the buffer
    gltf["buffers"] = [{"byteLength": len(blob), "uri": "data:;base64," + base64.b64encode(blob).decode()}]
    overrun = tmp_path / "overrun.gltf"
    overrun.write_text(json.dumps(gltf))
    with pytest.raises(RuntimeError, match="past its buffer"):
        rb.Mesh.load_gltf(overrun)


@pytest.mark.gpu
def test_gltf_scene_renders(tmp_path):
    path, _, _ = write(tmp_path, "glb")
    mesh = rb.Mesh.load_gltf(path)
    settings = rb.default_settings(mesh)
    renderer = rb.Renderer(settings)
    renderer.set_scene(mesh)
    frame = rb.frame_input(mesh, 64, 48)
    for _ in range(3):
        renderer.render(frame)
    image = renderer.display_image()
    assert image.shape == (48, 64, 4)
    hdr = renderer.download("display.hdr", np.float16)[:64 * 48 * 4].reshape(48, 64, 4)
    assert np.all(np.isfinite(hdr[..., :3].astype(np.float32)))
    # geometry covers part of the view, lit by the emissive triangle and the point light
    assert (hdr[..., 3] > 0.5).sum() > 100
    assert hdr[..., :3].astype(np.float32).max() > 0.0
