"""Shared test set-up: scenes, frame uniforms and buffers for the CUDA passes
(torch tensors on cuda:0) and for the oracle (numpy arrays)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

import restir_b200 as rb
from restir_b200.abi import (RestirDiReservoirs, RestirGBuffer, RestirGiHistory, RestirGiReservoirs, RestirParams,
                             RestirScene)


@dataclass
class SceneSetup:
    mesh: rb.Mesh
    bvh: rb.Bvh
    lights: rb.Lights
    settings: object
    materials: np.ndarray  # (m, 8)
    bvh_data: np.ndarray = None
    node_count: int = 0
    triangle_offset: int = 0
    keep: list = field(default_factory=list)

    def host_scene(self) -> RestirScene:
        s = RestirScene()
        data = self.bvh_data if self.bvh_data is not None else self.bvh.data
        s.bvh = data.ctypes.data
        s.node_count = self.node_count or self.bvh.desc.node_count
        s.triangle_offset = self.triangle_offset or self.bvh.desc.triangle_offset
        s.triangle_count = self.bvh.desc.triangle_count
        s.lights = self.lights.data.ctypes.data
        s.light_count = self.lights.count
        s.triangle_normals = self.bvh.triangle_normals.ctypes.data
        s.materials = self.materials.ctypes.data
        s.material_count = len(self.materials)
        return s

    def device_scene(self) -> RestirScene:
        import torch
        data = self.bvh_data if self.bvh_data is not None else self.bvh.data
        tensors = [torch.from_numpy(a).cuda() for a in (data, self.lights.data, self.bvh.triangle_normals,
                                                         self.materials.reshape(-1))]
        self.keep.extend(tensors)
        s = RestirScene()
        s.bvh = tensors[0].data_ptr()
        s.node_count = self.node_count or self.bvh.desc.node_count
        s.triangle_offset = self.triangle_offset or self.bvh.desc.triangle_offset
        s.triangle_count = self.bvh.desc.triangle_count
        s.lights = tensors[1].data_ptr()
        s.light_count = self.lights.count
        s.triangle_normals = tensors[2].data_ptr()
        s.materials = tensors[3].data_ptr()
        s.material_count = len(self.materials)
        return s


def make_scene(kind: int = rb.SCENE_CORNELL, seed: int = 0, triangles: int = 0, extra_lights: int = 0) -> SceneSetup:
    mesh = rb.Mesh.procedural(kind, seed, triangles)
    bvh = rb.Bvh(mesh)
    settings = rb.default_settings(mesh)
    settings.extra_lights = extra_lights
    lights = rb.Lights(bvh, mesh, settings)
    materials = np.ctypeslib.as_array(C.cast(mesh.desc.materials, C.POINTER(C.c_float)),
                                      (mesh.desc.material_count * 8,)).copy().reshape(-1, 8)
    return SceneSetup(mesh, bvh, lights, settings, materials)


def params_for(setup: SceneSetup, width: int, height: int, state=None, **overrides) -> tuple[RestirParams, object]:
    s = setup.settings
    for k, v in overrides.items():
        setattr(s, k, v)
    fi = rb.frame_input(setup.mesh, width, height)
    params, plan = rb.frame_params(s, setup.mesh, setup.lights.count, setup.bvh, fi,
                                   state if state is not None else rb.initial_state())
    return params, plan


# --- buffers ---------------------------------------------------------------------------------------

GBUFFER_FIELDS = (("albedo", np.uint8, 4), ("normal", np.uint8, 4), ("emissive", np.uint16, 4),
                  ("shading_normal", np.uint8, 4), ("depth", np.float32, 1))


def host_gbuffer(w: int, h: int) -> dict:
    return {name: np.zeros(w * h * c, dt) for name, dt, c in GBUFFER_FIELDS}


def gbuffer_struct(buffers: dict) -> RestirGBuffer:
    g = RestirGBuffer()
    for name, _, _ in GBUFFER_FIELDS:
        setattr(g, name, rb.ptr(buffers[name]))
    return g


def to_device(buffers: dict) -> dict:
    import torch
    return {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in buffers.items()}


def to_host(buffers: dict) -> dict:
    return {k: v.cpu().numpy() for k, v in buffers.items()}


def gi_reservoirs(buffers: dict, prefix: str = "") -> RestirGiReservoirs:
    r = RestirGiReservoirs()
    r.sample = rb.ptr(buffers[prefix + "sample"])
    r.receiver = rb.ptr(buffers[prefix + "receiver"])
    r.normal = rb.ptr(buffers[prefix + "normal"])
    return r


def gi_history(buffers: dict) -> RestirGiHistory:
    h = RestirGiHistory()
    h.sample = rb.ptr(buffers["sample"])
    h.receiver = rb.ptr(buffers["receiver"])
    h.normal = rb.ptr(buffers["normal"])
    h.color = rb.ptr(buffers["color"])
    h.moments = rb.ptr(buffers["moments"])
    return h


def di_reservoirs(buffers: dict) -> RestirDiReservoirs:
    r = RestirDiReservoirs()
    r.sample = rb.ptr(buffers["sample"])
    r.receiver = rb.ptr(buffers["receiver"])
    r.normal = rb.ptr(buffers["normal"])
    return r


def seeded_rays(setup: SceneSetup, n: int, seed: int = 0, tmax_scale: float = 4.0) -> np.ndarray:
    """Rays from random points in the scene bounds, directions uniform on the sphere: (n, 8) float32."""
    rng = np.random.default_rng(seed)
    lo = np.array(setup.mesh.desc.bounds_min, np.float32)
    hi = np.array(setup.mesh.desc.bounds_max, np.float32)
    o = lo + (hi - lo) * rng.random((n, 3), dtype=np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = tmax_scale * setup.mesh.desc.radius
    rays[:, 4:7] = d
    # A quarter of the rays are axis-parallel, the slab test's corner case.
    k = n // 4
    axis = rng.integers(0, 3, size=k)
    rays[:k, 4:7] = 0.0
    rays[np.arange(k), 4 + axis] = np.where(rng.random(k) < 0.5, -1.0, 1.0)
    return rays


def grid_cells(grid: np.ndarray, table_size: int, capacity: int) -> dict:
    """checksum -> (count, entries listed) of every occupied slot."""
    checks = grid[:table_size]
    counts = grid[table_size:2 * table_size]
    entries = grid[2 * table_size:].reshape(table_size, capacity)
    cells = {}
    for slot in np.nonzero(checks)[0]:
        c = int(counts[slot])
        cells[int(checks[slot])] = (c, entries[slot, :min(c, capacity)].copy())
    return cells


# --- display passes (include/restir_display.h) -------------------------------------------------------------------

def perspective_view_proj(eye, target, aspect: float, fov_y: float = 1.0, near: float = 0.05, far: float = 50.0):
    """A row-major view-projection (clip = M v, NDC depth in [0, 1]) and its inverse, float32."""
    eye = np.asarray(eye, np.float64)
    forward = np.asarray(target, np.float64) - eye
    forward /= np.linalg.norm(forward)
    right = np.cross(forward, [0.0, 1.0, 0.0])
    right /= np.linalg.norm(right)
    up = np.cross(right, forward)
    view = np.eye(4)
    view[0, :3], view[1, :3], view[2, :3] = right, up, forward
    view[:3, 3] = -view[:3, :3] @ eye
    f = 1.0 / np.tan(fov_y / 2.0)
    proj = np.zeros((4, 4))
    proj[0, 0], proj[1, 1] = f / aspect, f
    proj[2, 2], proj[2, 3] = far / (far - near), -near * far / (far - near)
    proj[3, 2] = 1.0
    vp = proj @ view
    return vp.astype(np.float32), np.linalg.inv(vp).astype(np.float32)


def half_image(values: np.ndarray) -> np.ndarray:
    """float (h, w, 4) -> RGBA16F bits (h * w * 4 uint16)."""
    return np.ascontiguousarray(values.astype(np.float16)).view(np.uint16).reshape(-1)


def display_inputs(width: int, height: int, seed: int = 0, specials: bool = True):
    """Seeded display-pass inputs: an HDR composite with background pixels
    (alpha 0), a depth buffer (1 on the background), last frame's TAA output,
    and matrices of a camera that moved a little since last frame."""
    rng = np.random.default_rng(seed)
    hdr = np.empty((height, width, 4), np.float32)
    hdr[..., :3] = rng.lognormal(-1.0, 1.5, (height, width, 3))
    background = rng.random((height, width)) < 0.15
    hdr[..., 3] = np.where(background, 0.0, 1.0)
    depth = np.where(background, 1.0, rng.uniform(0.90, 0.999, (height, width))).astype(np.float32)
    if specials:
        hdr[0, 0, :3] = np.inf
        hdr[height // 2, width // 3, 1] = np.nan
        hdr[height - 1, width - 1, :3] = 6.0e4
    history = np.empty((height, width, 4), np.float32)
    history[..., :3] = rng.lognormal(-1.0, 1.5, (height, width, 3))
    history[..., 3] = hdr[..., 3]
    aspect = width / height
    vp, inv = perspective_view_proj([0.3, 0.5, -3.0], [0.0, 0.0, 0.0], aspect)
    previous, _ = perspective_view_proj([0.33, 0.49, -3.02], [0.01, 0.0, 0.0], aspect)
    return {"hdr": half_image(hdr), "depth": depth.reshape(-1), "history": half_image(history),
            "inv_view_proj": inv, "previous_view_proj": previous, "view_proj": vp}


def display_params(width: int, height: int, inputs: dict, **fields):
    from restir_b200.abi import RestirDisplayParams
    p = RestirDisplayParams()
    p.inv_view_proj[:] = [float(v) for v in inputs["inv_view_proj"].reshape(-1)]
    p.previous_view_proj[:] = [float(v) for v in inputs["previous_view_proj"].reshape(-1)]
    p.width, p.height = width, height
    p.taa_history_valid = 1.0
    p.exposure_adapt = 0.05
    p.tonemapper = 1.0
    p.taa = 1.0
    for name, value in fields.items():
        setattr(p, name, value)
    return p
