"""Generates the known-answer fixtures in tests/golden/.

The reference has no tests or golden vectors of its own, so these pin the
oracle in two independent ways:

  hash_kat.json      PCG (shaders/hashgrid.sh:61-67, restir.sh:122-127) and
                     the xxHash32 avalanche (hashgrid.sh:69-78), restated here
                     in Python integer arithmetic.
  grid_keys.npz      gridCellSize / gridJitter / gridKey (hashgrid.sh:82-127)
                     for seeded positions and normals, restated here with
                     numpy float32 operations in the shader's order (one
                     rounding per operation, as the ABI's numeric conventions
                     fix it).
  reference_cornell.npz
                     the BVH buffer and light list that the reference's own
                     src/bvh.cpp and src/lights.cpp produce for the procedural
                     Cornell box (oracle/_ref, compiled from the reference's
                     sources; run in the container that has them).

Run: python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

M32 = 0xFFFFFFFF
f32 = np.float32


def pcg(v: int) -> int:
    state = (v * 747796405 + 2891336453) & M32
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & M32
    return ((word >> 22) ^ word) & M32


def xxhash_avalanche(v: int) -> int:
    v ^= v >> 15
    v = (v * 2246822519) & M32
    v ^= v >> 13
    v = (v * 3266489917) & M32
    v ^= v >> 16
    return v


def hash_kat() -> dict:
    rng = np.random.default_rng(0)
    inputs = [0, 1, 2, 3, 255, 65535, 0x5bd1e995, 0x68e31da4, 0x9e3779b9, M32 - 1, M32]
    inputs += [int(x) for x in rng.integers(0, 2**32, size=245, dtype=np.uint64)]
    return {"input": inputs, "pcg": [pcg(x) for x in inputs], "checksum": [xxhash_avalanche(x) for x in inputs]}


def normalize(v):
    return v * (f32(1.0) / np.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2], dtype=f32))


def cross(a, b):
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]], f32)


def grid_key(position, normal, camera, min_cell, pixel_size, cell_pixels, r0, r1, table_mask):
    offset = position - camera
    dist = np.sqrt(offset[0] * offset[0] + offset[1] * offset[1] + offset[2] * offset[2], dtype=f32)
    target = dist * pixel_size * cell_pixels
    ratio = max(target / min_cell, f32(1.0))
    level = int(np.frexp(ratio)[1]) - 1  # floor(log2) of a normal positive float
    cell = f32(min_cell * f32(2.0 ** level))
    if abs(normal[1]) < f32(0.99):
        tangent = normalize(cross(normal, np.array([0, 1, 0], f32)))
    else:
        tangent = normalize(cross(normal, np.array([1, 0, 0], f32)))
    bitangent = cross(normal, tangent)
    jittered = position + (tangent * (r0 - f32(0.5)) + bitangent * (r1 - f32(0.5))) * cell
    c = np.floor(jittered / cell).astype(np.int64)
    level_bits = int(np.array([cell], f32).view(np.uint32)[0])
    a = np.abs(normal)
    bucket = 4 if normal[2] >= 0 else 5
    if a[0] >= a[1] and a[0] >= a[2]:
        bucket = 0 if normal[0] >= 0 else 1
    elif a[1] >= a[2]:
        bucket = 2 if normal[1] >= 0 else 3
    cx, cy, cz = (int(v) & M32 for v in c)
    slot = pcg((level_bits + pcg((bucket + pcg((cx + pcg((cy + pcg(cz)) & M32)) & M32)) & M32)) & M32) & table_mask
    checksum = xxhash_avalanche(level_bits ^ xxhash_avalanche(bucket ^ xxhash_avalanche(
        cx ^ xxhash_avalanche(cy ^ xxhash_avalanche((cz + 0x9e3779b9) & M32)))))
    return level_bits, slot, max(checksum, 1)


def grid_keys() -> dict:
    rng = np.random.default_rng(3)
    n = 512
    positions = (rng.normal(size=(n, 3)) * 5.0).astype(f32)
    normals = rng.normal(size=(n, 3)).astype(f32)
    normals = np.stack([normalize(v) for v in normals]).astype(f32)
    normals[:16] = np.array([[0, 1, 0], [0, -1, 0], [1, 0, 0], [-1, 0, 0], [0, 0, 1], [0, 0, -1],
                             [0.7071068, 0.7071068, 0], [0, 0.995, 0.0998]] * 2, f32)
    randoms = rng.random((n, 2)).astype(f32)
    camera = np.array([1.5, 2.0, 7.0], f32)
    min_cell, pixel_size, cell_pixels, mask = f32(0.0198), f32(0.00165), f32(6.0), 65535
    out = np.array([grid_key(positions[i], normals[i], camera, min_cell, pixel_size, cell_pixels,
                             randoms[i, 0], randoms[i, 1], mask) for i in range(n)], np.uint64)
    return dict(positions=positions, normals=normals, randoms=randoms, camera=camera,
                constants=np.array([min_cell, pixel_size, cell_pixels], f32), table_mask=np.uint32(mask),
                cell_bits=out[:, 0].astype(np.uint32), slot=out[:, 1].astype(np.uint32),
                checksum=out[:, 2].astype(np.uint32))


def reference_cornell() -> dict:
    import ctypes as C

    import oracle.binding as ob
    import restir_b200 as rb
    mesh = rb.Mesh.procedural(rb.SCENE_CORNELL)
    positions = mesh.positions()
    tm = np.ctypeslib.as_array(C.cast(mesh.desc.triangle_material, C.POINTER(C.c_uint32)),
                               (mesh.triangle_count,)).copy()
    materials = np.ctypeslib.as_array(C.cast(mesh.desc.materials, C.POINTER(C.c_float)),
                                      (mesh.desc.material_count * 8,)).copy().reshape(-1, 8)
    data, nodes, offset, depth = ob.reference_bvh(positions, tm, materials)
    lights, count, triangles = ob.reference_lights(16, 0.3, 7, mesh.desc.bounds_min, mesh.desc.bounds_max,
                                                   (mesh.desc.radius / 1.75) ** 2)
    return dict(positions=positions, triangle_material=tm, materials=materials, bvh=data,
                header=np.array([nodes, offset, depth], np.uint32), lights=lights,
                light_header=np.array([count, triangles], np.uint32))


if __name__ == "__main__":
    (HERE / "hash_kat.json").write_text(json.dumps(hash_kat()))
    np.savez_compressed(HERE / "grid_keys.npz", **grid_keys())
    import oracle.binding as ob
    if ob.reference_available():
        np.savez_compressed(HERE / "reference_cornell.npz", **reference_cornell())
    else:
        print("oracle/_ref not built: reference_cornell.npz kept as it is")
    print("written to", HERE)
