"""Benchmark: one frame of the per-frame light-transport path at 1920x1080.

Workload (the metric's configuration): a seeded procedural scene of ~1M
triangles (boxes, 512-triangle spheres, thin two-sided planes, 128 emissive
panels), rendered at 1920x1080 with the reference's default settings: half-
resolution ReSTIR GI (2 candidates, 2 temporal and 4 spatial taps through the
world-space hash grid), ReSTIR DI at full resolution (8 candidates, 3 spatial
taps) over the 256 emissive triangles and 64 extra point lights, a 3x512^2
shadow atlas, the SVGF denoiser with 5 a-trous iterations, the composite.
A step is one frame through the C++ frame driver (restir_renderer_render).
The scene's buffers (126 MB of BVH, ~500 MB of frame targets) exceed the 126
MB L2, so no flush is needed between frames.

Reported: ms per frame (device time, CUDA events on the renderer's stream,
max over ranks), Mrays/s (rays counted on a separate profiling frame), the
relative MSE of the displayed frame against an FP64 progressive reference of
the same view, per-pass times, the roofline of the dominant pass, an end-to-
end time through the public API, and the CPU baseline (the oracle's
restatement of the same passes, on a bounded sample).

Multi-GPU: the path does not shard within a view (reuse reads any pixel's
reservoir through the world-space grid), so N ranks run N independent
replicas (weak scaling); value is the whole job's time per frame.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "1080p ms/frame at equal relMSE vs FP64 ref: plain vs radiance-cache; Mrays/s"
WIDTH, HEIGHT = 1920, 1080
TRIANGLES = 1_000_000
EXTRA_LIGHTS = 64
# The FP64 reference of the view: 1,024 frames (a 64-frame reference of this many-light view is far from
# converged: two 32-frame halves differ by a relative MSE of 30, which swamps the method's own error).
REFERENCE_FRAMES = 1024
ERROR_FRAMES = 120         # frames the relMSE and bias are averaged over
# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) per frame of the GI temporal pass's
# three kernels on this workload, one launch each, captured from the current build.
DOMINANT_TRAFFIC = {"gi_temporal": 165.4e6}
SIDE_STREAM_PASSES = ("shadow", "specular")
CACHE_TRAIN_FRAMES = 60    # online training before the radiance-cache form is timed
WORKLOAD = ("1920x1080 frame, seeded 1M-triangle city scene, GI 1/2 res + DI + specular GI + SVGF x5 + TAA + AgX "
            "tone mapping")

# Algorithmic (compulsory) bytes per pixel of each pass's image reads and
# writes, besides its BVH traversal (32 B per node fetch, 48 B per triangle
# test, counted on the device in a profiling frame): the G-buffer, reservoir,
# history and target texels each pass must read or write once.
PASS_PIXEL_BYTES = {
    "shadow": ("atlas", 4),
    "gbuffer": ("full", 24),
    "di_temporal": ("full", 96),
    "di_spatial": ("full", 72),
    "grid": ("gi", 20),
    "gi_temporal": ("gi", 116),
    "gi_spatial": ("gi", 124),
    "denoise": ("gi", 56 + 5 * 48),
    "composite": ("full", 50),
    "reference": ("full", 57),
    # radiance-cache training: per training sample a query and a target (80 B) and the hash-grid
    # gather of two queries (2 x 512 B); counted per GI pixel only when it runs
    "cache": ("none", 0),
    # TAA + tone mapping, fused: the composite (3x3 neighbourhood, read once), depth, the TAA history,
    # the TAA target and the BGRA8 display (8 + 4 + 8 + 8 + 4); the exposure's 4,096 samples are noise
    "display": ("full", 32),
    # indirect specular: G-buffer 12, history receiver and normal 32, specular history 8 and target 8,
    # last frame's HDR at the hit 8
    "specular": ("gi", 68),
}


def gather_probe(renderer, repeats: int = 5) -> float:
    """GB/s of random 32-byte row gathers from the scene's BVH nodes
    (restir_gather_probe; the node rows fit the L2, where the traversal
    kernels find them), on the renderer's stream."""
    import torch
    import restir_b200 as rb
    lib = rb.load()
    pointer, nbytes = renderer.buffer("bvh")
    params, _, _ = renderer.last_frame()
    rows = min(int(nbytes // 32), 61_000_000 // 32)  # the node part of the buffer, at most 61 MB
    blocks, gathers = 148 * 8, 256
    out = torch.empty(blocks * 256, dtype=torch.float32, device="cuda")
    stream = torch.cuda.ExternalStream(renderer.stream)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for r in range(repeats + 2):
        if r == 2:
            start.record(stream)
        rb.check(lib.restir_gather_probe(pointer, rows, blocks, gathers, r, out.data_ptr(), renderer.stream),
                 "gather probe")
    stop.record(stream)
    torch.cuda.synchronize()
    fetched = blocks * 256 * gathers * 32 * repeats
    return fetched / (start.elapsed_time(stop) * 1e-3) / 1e9


def accumulate_reference(renderer, frame, frames: int = REFERENCE_FRAMES) -> dict:
    """The FP64 progressive reference of the view (reference mode, `frames`
    frames), and its own noise: the relative MSE and bias between its two
    halves (frames 1..n/2 and n/2+1..n), each a reference of n/2 frames;
    the whole reference's error against the converged image is about a
    quarter of that relative MSE."""
    n = frame.width * frame.height
    renderer.set_reference_accumulation(True)
    half = None
    for i in range(frames):
        renderer.render(frame)
        if i + 1 == frames // 2:
            half = renderer.download("reference.mean", np.float64)[:3 * n].copy()
    full = renderer.download("reference.mean", np.float64)[:3 * n].copy()
    alpha = renderer.download("reference.alpha", np.uint8)[:n] > 0
    renderer.set_reference_accumulation(False)
    with np.errstate(invalid="ignore", over="ignore"):
        second = 2.0 * full - half

    def luminance(mean):
        return 0.2126 * mean[:n] + 0.7152 * mean[n:2 * n] + 0.0722 * mean[2 * n:]
    with np.errstate(invalid="ignore", over="ignore"):
        a, b = luminance(half)[alpha], luminance(second)[alpha]
    finite = np.isfinite(a) & np.isfinite(b)
    a, b = a[finite], b[finite]
    return {"frames": frames, "split_half_rel_mse": float(np.mean((a - b) ** 2 / (b * b + 0.01))),
            "split_half_bias": float(a.mean() / b.mean() - 1.0)}


def load_peaks() -> tuple[float, str]:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, value in zip(names, parts[5:9]):
                if value.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def scene_and_settings(rb, triangles: int = TRIANGLES):
    mesh = rb.Mesh.procedural(rb.SCENE_CITY, 0, triangles)
    settings = rb.default_settings(mesh)
    settings.extra_lights = EXTRA_LIGHTS
    return mesh, settings


def cpu_frames(steps: int, warmup: int) -> dict:
    """The reference's per-frame path on the host cores, full frames of the
    same workload: the seeded 1M-triangle city at 1920x1080 with the
    reference's default settings, its BVH and light list from the reference's
    own src/bvh.cpp and src/lights.cpp (oracle/_ref/libref_bvh.so), the frame
    uniforms from the oracle's restatement of renderer.cpp, and every compute
    and fragment pass the reference runs as a shader (grid insert, GI
    temporal and spatial, DI temporal and spatial, SVGF, composite, specular)
    from the reference's own shader code compiled as C++
    (oracle/_ref/libref_shaders.so); the G-buffer and shadow-atlas ray casts
    (the reference rasterizes them) and TAA and tone mapping come from the
    oracle. All host threads. Nothing of this repository's library is loaded.
    `warmup` untimed frames (history), then `steps` timed frames."""
    import oracle.binding as ob
    from oracle.frame import FrameRunner
    from oracle.workload import OracleSetup
    import restir_b200 as rb

    threads = os.cpu_count() or 1
    ob.load().oracle_set_threads(threads)
    ob.load_shaders().ref_set_threads(threads)
    t = time.perf_counter()
    setup = OracleSetup(rb.SCENE_CITY, 0, TRIANGLES, extra_lights=EXTRA_LIGHTS)
    setup_ms = (time.perf_counter() - t) * 1e3
    runner = FrameRunner(setup, WIDTH, HEIGHT, "ref", setup.settings)
    for _ in range(warmup):
        runner.render()
    times, pass_ms = [], {}
    for _ in range(steps):
        runner.prepare()
        start = time.perf_counter()
        for name, fn in runner.passes():
            t = time.perf_counter()
            fn()
            pass_ms[name] = pass_ms.get(name, 0.0) + (time.perf_counter() - t) * 1e3 / steps
        runner.finish()
        times.append((time.perf_counter() - start) * 1e3)
    return {"value": float(np.mean(times)), "unit": "ms/frame", "cores": threads, "kind": "reference",
            "sample": f"{steps} full {WIDTH}x{HEIGHT} frame(s) of the {setup.mesh.triangle_count}-triangle city after "
                      f"{warmup} history frame(s): the reference's shader code (compiled as C++) for its compute and "
                      f"fragment passes, its bvh.cpp/lights.cpp for the scene; ray-cast G-buffer and shadow atlas, TAA "
                      f"and tone mapping from the oracle",
            "frame_ms": [float(v) for v in times], "pass_ms": {k: float(v) for k, v in pass_ms.items()},
            "scene_setup_ms": setup_ms, "scene_triangles": int(setup.mesh.triangle_count)}


def reference_arm(args, rank: int, world: int) -> None:
    """--impl reference: the reference's per-frame path on the host cores
    (cpu_frames), one full frame per step. The reference runs the path as
    bgfx shaders; with no graphics stack here its own shader code runs on the
    CPU, compiled as C++. Under torchrun only rank 0 works."""
    if rank != 0:
        return
    result = cpu_frames(args.steps, args.warmup)
    value = result["value"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "ms/frame", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": value, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
        "config": {"workload": WORKLOAD, "scene_triangles": result["scene_triangles"], "width": WIDTH,
                   "height": HEIGHT},
        "cpu_baseline": {k: result[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "pass_ms": result["pass_ms"],
        "e2e": {"value": value, "unit": "ms/frame", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cache_kernels(args) -> None:
    """--cache-kernels: the radiance cache's kernels alone on seeded synthetic
    queries (the frame's query count, 2,073,600, and a 65,536-sample training
    batch), timed with CUDA events; for profiling the tcgen05 MLP."""
    import torch
    import restir_b200 as rb
    rng = np.random.default_rng(1)

    def queries(n):
        q = np.zeros((n, 16), np.float32)
        q[:, 0:3] = rng.uniform(-1.0, 1.0, (n, 3))
        q[:, 3] = rng.uniform(0.0, 1.0, n)
        for col in (4, 8):
            v = rng.normal(size=(n, 3))
            q[:, col:col + 3] = v / np.linalg.norm(v, axis=1, keepdims=True)
        q[:, 7] = 1.0
        q[:, 12:15] = rng.uniform(0.05, 0.95, (n, 3))
        return torch.from_numpy(q).cuda()

    cache = rb.RadianceCache(rb.cache_config(bounds_min=(-1.0, -1.0, -1.0), bounds_max=(1.0, 1.0, 1.0)))
    frame_queries = queries(2_073_600)
    train_queries = queries(65536)
    targets = torch.rand((65536, 4), device="cuda")
    targets[:, 3] = 1.0
    out = torch.empty((frame_queries.shape[0], 4), dtype=torch.float16, device="cuda")
    for _ in range(args.warmup):
        cache.query(frame_queries, out)
        cache.train(train_queries, targets)
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(args.steps):
        cache.query(frame_queries, out)
    stop.record()
    torch.cuda.synchronize()
    query_ms = start.elapsed_time(stop) / args.steps
    start.record()
    for _ in range(args.steps):
        cache.train(train_queries, targets)
    stop.record()
    torch.cuda.synchronize()
    train_ms = start.elapsed_time(stop) / args.steps
    flops = 2 * (64 * 64 * 4 + 16 * 64) * frame_queries.shape[0]
    print(json.dumps({"cache_kernels": True, "query_ms": query_ms, "queries": int(frame_queries.shape[0]),
                      "query_tflops": flops / (query_ms * 1e-3) / 1e12, "train_ms": train_ms,
                      "training_samples": 65536, "loss": cache.scalars().loss,
                      "status": rb.status_flags()}), flush=True)


def bvh_build(args) -> None:
    """--bvh-build: scene preparation, the BVH of the seeded city scene at 1M and
    4M triangles (the stress configuration's size) built on the device
    (restir_bvh_build_gpu) and on the host (16 threads), with a check that the
    two buffers are identical."""
    import restir_b200 as rb
    lines = {}
    for triangles in (TRIANGLES, 4 * TRIANGLES):
        mesh = rb.Mesh.procedural(rb.SCENE_CITY, 0, triangles)
        device_ms = []
        for step in range(args.warmup + args.steps):
            bvh = rb.Bvh(mesh, device=True)
            if step >= args.warmup:
                device_ms.append(bvh.desc.build_ms)
        host = rb.Bvh(mesh)
        identical = bool(np.array_equal(bvh.data.view(np.uint32), host.data.view(np.uint32))
                         and np.array_equal(bvh.order, host.order))
        lines[str(mesh.triangle_count)] = {"device_ms": float(np.median(device_ms)), "host_ms": host.desc.build_ms,
                                           "host_threads": os.cpu_count(), "nodes": int(host.desc.node_count),
                                           "identical": identical}
    print(json.dumps({"bvh_build": lines, "steps": args.steps, "warmup": args.warmup}), flush=True)


# The quality settings --pareto sweeps, each on top of the defaults.
PARETO_VARIANTS = [
    ("default", {}),
    ("candidates1", {"initial_candidates": 1}),
    ("spatial2", {"spatial_taps": 2}),
    ("candidates1_spatial2", {"initial_candidates": 1, "spatial_taps": 2}),
    ("no_specular", {"specular_gi": 0}),
    ("atrous3", {"atrous_iterations": 3}),
    ("cheapest", {"initial_candidates": 1, "spatial_taps": 2, "specular_gi": 0, "atrous_iterations": 3}),
    # the cache-only GI (no GI rays: the cache at each GI pixel's surface); radiance-cache form only
    ("cache_only", {"cache_only_gi": 1}),
    ("cache_only_no_specular", {"cache_only_gi": 1, "specular_gi": 0}),
    ("cache_only_more_training", {"cache_only_gi": 1, "cache_training_samples": 131072}),
    ("cache_only_lr3e-3", {"cache_only_gi": 1, "cache_learning_rate": 3e-3}),
    # diagnostic: no indirect light at all (how much of the error the GI term carries)
    ("no_gi", {"initial_candidates": 0, "temporal_taps": 0, "spatial_taps": 0, "specular_gi": 0}),
]
# (GI resolution is not swept: the FP64 reference is rendered at the view's GI
# resolution, so another divisor would be judged against another reference.)


def pareto(args) -> None:
    """--pareto: the metric's comparison at equal error. Both forms (plain and
    radiance cache) over PARETO_VARIANTS on the 1920x1080 city view, each pair
    from a fresh renderer (fresh history and, for the cache form, a fresh
    cache): the 1,024-frame FP64 reference with the default settings, then the
    variant's settings, warm-up (CACHE_TRAIN_FRAMES of training for the cache
    form), device ms/frame over `steps` frames (CUDA events) and the mean
    relMSE over ERROR_FRAMES frames; then, per form, the cheapest setting
    whose relMSE is within the plain default's."""
    import torch
    import restir_b200 as rb
    mesh, settings = scene_and_settings(rb)
    frame = rb.frame_input(mesh, WIDTH, HEIGHT)
    rows = []
    for form in ("plain", "cache"):
        for name, changes in PARETO_VARIANTS:
            if form == "plain" and changes.get("cache_only_gi"):
                continue
            renderer = rb.Renderer(settings)
            renderer.set_scene(mesh)
            accumulate_reference(renderer, frame)
            s = renderer.settings
            for field, value in changes.items():
                setattr(s, field, value)
            s.radiance_cache = 1 if form == "cache" else 0
            renderer.settings = s
            for _ in range(CACHE_TRAIN_FRAMES if form == "cache" else max(args.warmup, 20)):
                renderer.render(frame)
            stream = torch.cuda.ExternalStream(renderer.stream)
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            start.record(stream)
            for _ in range(args.steps):
                renderer.render(frame)
            stop.record(stream)
            torch.cuda.synchronize()
            ms = start.elapsed_time(stop) / args.steps
            error = error_stats(renderer, frame, ERROR_FRAMES)
            rows.append({"form": form, "variant": name, "ms_per_frame": ms, "rel_mse": error["mean"]})
            renderer.close()
    target = next(r["rel_mse"] for r in rows if r["form"] == "plain" and r["variant"] == "default")
    best = {}
    for form in ("plain", "cache"):
        ok = [r for r in rows if r["form"] == form and r["rel_mse"] <= target]
        best[form] = min(ok, key=lambda r: r["ms_per_frame"]) if ok else None
    ratio = (best["plain"]["ms_per_frame"] / best["cache"]["ms_per_frame"]) if best["plain"] and best["cache"] else None
    print(json.dumps({"pareto": rows, "target_rel_mse": target, "best": best,
                      "plain_over_cache_at_equal_rel_mse": ratio, "steps": args.steps}), flush=True)


def settings_fields(settings):
    """The (name, value) pairs of a RestirSettings (the variants start from these)."""
    return [(name, getattr(settings, name)) for name, _ in type(settings)._fields_
            if not hasattr(getattr(settings, name), "__len__")]


BATCH_SIZES = [(640, 360), (960, 540), (1280, 720), (1920, 1080), (800, 450), (1600, 900), (1024, 576), (1440, 810)]


def camera_path(rb, mesh, width: int, height: int, frames: int, seed: int = 0):
    """A seeded camera path: the eye moves through four seeded control points
    around the scene's default view (Catmull-Rom), yaw and pitch sway with
    it; one frame input per frame at 1/60 s."""
    rng = np.random.default_rng(seed)
    radius = mesh.desc.radius
    eye0 = np.array(mesh.desc.camera_eye, np.float64)
    points = eye0 + rng.uniform(-0.08, 0.08, (4, 3)) * radius
    points[:, 1] = eye0[1] + rng.uniform(-0.02, 0.04, 4) * radius
    yaws = mesh.desc.camera_yaw + rng.uniform(-0.25, 0.25, 4)
    pitches = mesh.desc.camera_pitch + rng.uniform(-0.05, 0.05, 4)
    inputs = []
    for i in range(frames):
        t = 3.0 * i / max(frames - 1, 1)
        k = min(int(t), 2)
        u = t - k

        def spline(v):
            p0, p1, p2, p3 = v[max(k - 1, 0)], v[k], v[k + 1], v[min(k + 2, 3)]
            return 0.5 * ((2 * p1) + (-p0 + p2) * u + (2 * p0 - 5 * p1 + 4 * p2 - p3) * u * u
                          + (-p0 + 3 * p1 - 3 * p2 + p3) * u ** 3)
        inputs.append(rb.frame_input(mesh, width, height, eye=[float(x) for x in spline(points)],
                                     yaw=float(spline(yaws)), pitch=float(spline(pitches))))
    return inputs


def mid_config(args) -> None:
    """--config mid: the mid configuration, a seeded courtyard of instanced boxes
    and arches (100k triangles, albedo U[0.2, 0.8], roughness U[0.05, 1]) with
    64 extra point lights beside its 256 emissive triangles, 1280x720, GI at
    half resolution with temporal and spatial reuse, ReSTIR DI, SVGF with 5
    a-trous levels, a 2^20-slot hash grid, 60 frames on a seeded camera path
    (device time per frame, CUDA events). Then, held at the path's last pose,
    the relative MSE and bias against a 1,024-frame FP64 reference."""
    import torch
    import restir_b200 as rb
    mesh = rb.Mesh.procedural(rb.SCENE_COURTYARD, 0, 100_000)
    renderer = rb.Renderer(rb.default_settings(mesh))
    renderer.set_scene(mesh, use_scene_defaults=True)
    settings = renderer.settings
    settings.extra_lights = 64
    settings.grid_table_size = 1 << 20
    renderer.settings = settings
    path = camera_path(rb, mesh, 1280, 720, 60)
    for _ in range(args.warmup):
        renderer.render(path[0])
    stream = torch.cuda.ExternalStream(renderer.stream)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    for frame in path:
        renderer.render(frame)
    stop.record(stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(stop) / len(path)
    pass_ms = renderer.pass_history(len(path)).mean(axis=0)
    final = path[-1]
    counts = renderer.profile_frame(final)
    reference = accumulate_reference(renderer, final)
    for _ in range(60):
        renderer.render(final)
    error = error_stats(renderer, final, 60)
    params, _, _ = renderer.last_frame()
    rays = int(counts[:, 0:3].sum())
    print(json.dumps({"config": "mid", "workload": "1280x720, seeded 100k-triangle courtyard, 64 point lights + "
                      "256 emissive triangles, GI 1/2 res + DI + specular GI + SVGF x5 + TAA, 2^20-slot grid, "
                      "60-frame seeded camera path", "scene_triangles": mesh.triangle_count,
                      "di_lights": params.di_light_count, "grid_table_size": params.grid_table_size,
                      "ms_per_frame": ms, "frames": len(path), "mrays_per_s": rays / (ms * 1e-3) / 1e6,
                      "rel_mse_vs_fp64_reference": error["mean"], "bias_vs_fp64_reference": error["bias"],
                      "reference_noise": reference, "truncated_rays_per_frame": int(counts[:, 7].sum()),
                      "pass_ms": {name: float(pass_ms[i]) for i, name in enumerate(rb.PASS_NAMES)},
                      "status": rb.status_flags()}), flush=True)
    renderer.close()


def stress_config(args) -> None:
    """--config stress: the stress configuration, 3840x2160 on the seeded
    4M-triangle city with 2,048 emissive panels (4,096 emissive triangles) and
    1,024 extra point lights orbiting on seeded circles, GI + DI + SVGF + the
    radiance cache (GI passes with the cache), a 2^22-slot hash grid, 240
    frames at 1/60 s (device time per frame, CUDA events). Then, with the
    lights held where they are (delta_time 0), the relative MSE and bias
    against a 4,096-frame FP64 reference (4,096 samples per pixel)."""
    import torch
    import restir_b200 as rb
    mesh = rb.Mesh.procedural(rb.SCENE_CITY_LIT, 0, 4_000_000)
    renderer = rb.Renderer(rb.default_settings(mesh))
    t = time.perf_counter()
    renderer.set_scene(mesh, use_scene_defaults=True)
    scene_ms = (time.perf_counter() - t) * 1e3
    settings = renderer.settings
    settings.extra_lights = 1024
    settings.grid_table_size = 1 << 22
    settings.radiance_cache = 1
    settings.extra_light_orbit = 0.5
    renderer.settings = settings
    frame = rb.frame_input(mesh, 3840, 2160)
    for _ in range(max(args.warmup, 3)):
        renderer.render(frame)
    stream = torch.cuda.ExternalStream(renderer.stream)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    frames = 240
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(frames):
        renderer.render(frame)
    stop.record(stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(stop) / frames
    pass_ms = renderer.pass_history(min(frames, 64)).mean(axis=0)
    held = rb.frame_input(mesh, 3840, 2160, delta_time=0.0)
    counts = renderer.profile_frame(held)
    reference = accumulate_reference(renderer, held, 4096)
    for _ in range(120):
        renderer.render(held)
    # A few reference pixels overflow half precision (extra lights right at a surface): the
    # composite stores inf, which the reference's mean keeps (its guard is for NaN only,
    # fs_reference.sc:22-23), so the error pass's sums are not finite. The relative MSE and
    # bias are therefore taken on the host over the pixels whose reference is finite.
    n = 3840 * 2160
    mean = renderer.download("reference.mean", np.float64)[:3 * n]
    alpha = renderer.download("reference.alpha", np.uint8)[:n] > 0
    lr = 0.2126 * mean[:n] + 0.7152 * mean[n:2 * n] + 0.0722 * mean[2 * n:]
    finite = alpha & np.isfinite(lr)
    values, biases = [], []
    for _ in range(30):
        renderer.render(held)
        image = renderer.download("display.hdr", np.float16)[:4 * n].reshape(n, 4).astype(np.float64)
        li = 0.2126 * image[:, 0] + 0.7152 * image[:, 1] + 0.0722 * image[:, 2]
        ok = finite & np.isfinite(li)
        values.append(float(np.mean((li[ok] - lr[ok]) ** 2 / (lr[ok] ** 2 + 0.01))))
        biases.append(float(li[ok].mean() / lr[ok].mean() - 1.0))
    error = {"mean": float(np.mean(values)), "bias": float(np.mean(biases)),
             "pixels_excluded": int(np.count_nonzero(alpha & ~np.isfinite(lr)))}
    params, _, _ = renderer.last_frame()
    rays = int(counts[:, 0:3].sum())
    print(json.dumps({"config": "stress", "workload": "3840x2160, seeded 4M-triangle city, 1,024 orbiting point "
                      "lights + 4,096 emissive triangles, GI 1/2 res with the radiance cache + DI + specular GI + "
                      "SVGF x5 + TAA, 2^22-slot grid, 240 frames", "scene_triangles": mesh.triangle_count,
                      "scene_setup_ms": scene_ms, "di_lights": params.di_light_count,
                      "grid_table_size": params.grid_table_size, "ms_per_frame": ms, "frames": frames,
                      "mrays_per_s": rays / (ms * 1e-3) / 1e6, "rel_mse_vs_fp64_reference": error["mean"],
                      "bias_vs_fp64_reference": error["bias"], "reference_noise": reference,
                      "error_pixels_excluded_nonfinite_reference": error["pixels_excluded"],
                      "truncated_rays_per_frame": int(counts[:, 7].sum()),
                      "pass_ms": {name: float(pass_ms[i]) for i, name in enumerate(rb.PASS_NAMES)},
                      "status": rb.status_flags()}), flush=True)
    renderer.close()


def batched(args) -> None:
    """--batched: the batched form, 8 views of uneven resolution (640x360 to
    1920x1080, each its own camera) of the 1M-triangle scene in one frame
    (restir_batch_*: one scene, one shadow atlas, one GI ray queue and tracer
    launch, one CUDA graph); the tracer shape from the autotuner. Beside it the
    same views rendered one after another by one renderer."""
    import torch
    import restir_b200 as rb
    mesh, settings = scene_and_settings(rb)
    base = rb.frame_input(mesh, 64, 64)
    inputs = [rb.frame_input(mesh, w, h, yaw=base.yaw + 0.3 * v, pitch=base.pitch)
              for v, (w, h) in enumerate(BATCH_SIZES)]
    batch = rb.Batch(settings, len(inputs))
    batch.set_scene(mesh)
    best = batch.autotune(inputs, frames=5)
    for _ in range(args.warmup):
        batch.render(inputs)
    batch.synchronize()
    stream = torch.cuda.ExternalStream(batch.stream)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        batch.render(inputs)
    stop.record(stream)
    torch.cuda.synchronize()
    batch_ms = start.elapsed_time(stop) / args.steps
    batch.close()
    single = rb.Renderer(settings)
    single.set_scene(mesh)
    sequential = []
    sstream = torch.cuda.ExternalStream(single.stream)
    for frame in inputs:
        for _ in range(args.warmup):
            single.render(frame)
        single.synchronize()
        start.record(sstream)
        for _ in range(args.steps):
            single.render(frame)
        stop.record(sstream)
        torch.cuda.synchronize()
        sequential.append(start.elapsed_time(stop) / args.steps)
    single.close()
    pixels = sum(w * h for w, h in BATCH_SIZES)
    print(json.dumps({"batched": True, "views": [f"{w}x{h}" for w, h in BATCH_SIZES], "ms_per_batch_frame": batch_ms,
                      "mpixels_per_s": pixels / (batch_ms * 1e-3) / 1e6, "sequential_ms": float(sum(sequential)),
                      "sequential_per_view_ms": sequential, "speedup_vs_sequential": float(sum(sequential)) / batch_ms,
                      "tuning": {"tracer_threads": best.tracer_threads,
                                 "tracer_blocks_per_sm": best.tracer_blocks_per_sm,
                                 "autotune_ms_per_frame": best.ms_per_frame},
                      "status": rb.status_flags()}), flush=True)


def max_over_ranks(values, dist, device: str) -> list:
    """Every rank's timings reduced to the maximum over the ranks (the job's
    time is its slowest replica's); every rank must call it. dist None: one
    process."""
    import torch
    total = torch.tensor(values, device=device, dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(total, op=dist.ReduceOp.MAX)
    return [float(v) for v in total]


def error_stats(renderer, frame, frames: int) -> dict:
    """relMSE of the live image against the FP64 reference over `frames` frames."""
    values, biases = [], []
    for _ in range(frames):
        renderer.render(frame)
        metrics = renderer.frame_submitted()
        values.append(metrics.relative_mse)
        biases.append(metrics.bias)
    return {"mean": float(np.mean(values)), "median": float(np.median(values)), "bias": float(np.mean(biases))}


def cache_arm(renderer, frame, steps: int, changes: dict | None = None) -> dict:
    """The radiance-cache form on the same view (with `changes` to the settings
    on top, restored after): CACHE_TRAIN_FRAMES frames of online training,
    then `steps` timed frames (CUDA events on the renderer's stream) and the
    relMSE over ERROR_FRAMES frames."""
    import torch
    import restir_b200 as rb
    settings = renderer.settings
    saved = {name: getattr(settings, name) for name in (changes or {})}
    settings.radiance_cache = 1
    for name, value in (changes or {}).items():
        setattr(settings, name, value)
    renderer.settings = settings
    for _ in range(CACHE_TRAIN_FRAMES):
        renderer.render(frame)
    renderer.synchronize()
    stream = torch.cuda.ExternalStream(renderer.stream)
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(steps):
        renderer.render(frame)
    stop.record(stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(stop) / steps
    pass_ms = renderer.pass_history(steps)
    mean_pass = pass_ms.mean(axis=0) if len(pass_ms) else np.zeros(len(rb.PASS_NAMES))
    error = error_stats(renderer, frame, ERROR_FRAMES)
    params, _, _ = renderer.last_frame()
    settings.radiance_cache = 0
    for name, value in saved.items():
        setattr(settings, name, value)
    renderer.settings = settings
    return {"ms_per_frame": ms, "settings": dict(changes or {}), "rel_mse_vs_fp64_reference": error["mean"],
            "rel_mse_median": error["median"], "bias_vs_fp64_reference": error["bias"],
            "training_frames": CACHE_TRAIN_FRAMES + steps, "training_samples_per_frame": int(params.cache_training_samples),
            "pass_ms": {name: float(mean_pass[i]) for i, name in enumerate(rb.PASS_NAMES)}}


def own_arm(args, rank: int, world: int) -> None:
    import torch

    import restir_b200 as rb

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_module
        dist = dist_module
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    if args.quick and args.small:
        # A small case of the same kind of frame, for ncu captures of one kernel.
        mesh, settings = scene_and_settings(rb, 100_000)
    else:
        mesh, settings = scene_and_settings(rb)
    renderer = rb.Renderer(settings)
    t = time.perf_counter()
    renderer.set_scene(mesh, use_scene_defaults=True)
    scene_ms = (time.perf_counter() - t) * 1e3
    settings = renderer.settings
    settings.extra_lights = EXTRA_LIGHTS
    renderer.settings = settings
    frame = rb.frame_input(mesh, WIDTH, HEIGHT)

    if args.quick:
        # Profiling runs: W warm-up frames, then K frames, nothing else.
        if args.radiance_cache or args.set:
            settings = renderer.settings
            settings.radiance_cache = 1 if args.radiance_cache else settings.radiance_cache
            for item in args.set:
                name, value = item.split("=")
                setattr(settings, name, type(getattr(settings, name))(float(value)))
            renderer.settings = settings
        for _ in range(args.warmup):
            renderer.render(frame)
        for _ in range(args.steps):
            renderer.render(frame)
        renderer.synchronize()
        print(json.dumps({"quick": True, "frames": args.warmup + args.steps}), flush=True)
        renderer.close()
        return

    # FP64 progressive reference of this view (not timed).
    reference = accumulate_reference(renderer, frame)

    # Let the live history settle, then one profiling frame for the work counts.
    for _ in range(max(args.warmup, 3)):
        renderer.render(frame)
    counts = renderer.profile_frame(frame)
    for _ in range(args.warmup):
        renderer.render(frame)
    renderer.synchronize()

    sampler = ClockSampler(local)
    sampler.start()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.ExternalStream(renderer.stream)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(args.steps):
        renderer.render(frame, graph=args.graph)
    stop.record(stream)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    elapsed_ms = start.elapsed_time(stop)
    clocks = sampler.stop()
    pass_ms = renderer.pass_history(args.steps) if not args.graph else np.zeros((0, len(rb.PASS_NAMES)))
    metrics = renderer.frame_submitted()
    # The timed frames' plan (the radiance-cache arms below change the settings).
    params, plan, _ = renderer.last_frame()

    # End to end through the public API: each step renders the frame from its
    # host-side input and reads the frame's error record back to the host.
    renderer.synchronize()
    t = time.perf_counter()
    for _ in range(args.steps):
        renderer.render(frame)
        step_metrics = renderer.frame_submitted()
    e2e_ms = (time.perf_counter() - t) * 1e3 / args.steps

    # relMSE against the FP64 reference over several frames (one frame's value
    # swings with the fireflies of the specular DI), then the same for the
    # radiance-cache form after it has trained.
    plain_error = error_stats(renderer, frame, ERROR_FRAMES)
    cache_line = cache_arm(renderer, frame, args.steps) if not args.no_cache else None
    # The cache-only GI form at its cheapest setting of the --pareto sweep (the
    # cache continues from the form above).
    cache_only_line = (cache_arm(renderer, frame, args.steps, {"cache_only_gi": 1, "specular_gi": 0})
                       if not args.no_cache else None)

    elapsed_ms, e2e_ms = max_over_ranks([elapsed_ms, e2e_ms], dist, "cuda")
    if rank != 0:
        renderer.close()
        if dist is not None:
            dist.destroy_process_group()
        return

    ms_per_frame = elapsed_ms / args.steps
    # BVH rays: primary and shadow-map ray casts, GI closest-hit rays, visibility rays (depth-buffer
    # marches are reported beside them, not counted as rays).
    rays = int(counts[:, 0:3].sum())
    passes = rb.PASS_NAMES
    mean_pass = pass_ms.mean(axis=0) if len(pass_ms) else np.zeros(len(passes))
    sizes = {"full": WIDTH * HEIGHT, "gi": params.gi_width * params.gi_height,
             "atlas": 6 * params.shadow_face_size ** 2, "none": 0}
    _, bvh_bytes = renderer.buffer("bvh")
    image_bytes, fetched_bytes, pass_bytes = {}, {}, {}
    for i, name in enumerate(passes):
        res, per_pixel = PASS_PIXEL_BYTES[name]
        ran = mean_pass[i] > 0
        image_bytes[name] = (sizes[res] * per_pixel + (8 * params.grid_table_size if name == "grid" else 0)) if ran else 0
        fetched_bytes[name] = (32 * int(counts[i, 4]) + 48 * int(counts[i, 5])) if ran else 0
        pass_bytes[name] = image_bytes[name] + fetched_bytes[name]
    mean_pass = [float(v) for v in mean_pass]
    # The dominant pass of the main chain: the shadow atlas and the specular pass
    # run on a second, lower-priority stream, so their event intervals include
    # the time they wait behind the chain for free SMs.
    chain = [i for i, name in enumerate(passes) if name not in SIDE_STREAM_PASSES]
    dominant = max(chain, key=lambda i: mean_pass[i])
    name = passes[dominant]
    seconds = mean_pass[dominant] * 1e-3
    peak, peak_kind = load_peaks()
    # Compulsory HBM bytes of the pass: its image reads and writes, and each BVH row it touches
    # at most once (no more than the whole BVH).
    footprint = image_bytes[name] + min(fetched_bytes[name], bvh_bytes)
    achieved = float(footprint / seconds / 1e9) if seconds > 0 else 0.0
    l2_gather_gbs = gather_probe(renderer)
    fetched_gbs = float(fetched_bytes[name] / seconds / 1e9) if seconds > 0 else 0.0
    share = {name: (mean_pass[i] / ms_per_frame if ms_per_frame > 0 else 0.0) for i, name in enumerate(passes)}
    # shadow, G-buffer, DI x2, grid x2, GI temporal (3 kernels as a wavefront), GI spatial, denoiser, composite,
    # display (auto exposure when on, then TAA + tone mapping), specular (3 kernels as a wavefront)
    gi_temporal_kernels = 3 if settings.wavefront else 1
    launches = (2 + (2 if plan.di_active else 0) + 2 + gi_temporal_kernels + 1
                + (1 + plan.atrous_iterations if plan.denoiser else 0) + 1
                + ((1 + plan.exposure) if plan.display else 0)
                + ((3 if settings.wavefront else 1) if plan.specular else 0))

    if args.no_cpu_baseline:
        baseline = None
    else:
        frames = cpu_frames(steps=1, warmup=1)
        baseline = {k: frames[k] for k in ("value", "unit", "cores", "kind", "sample", "pass_ms")}
    line = {
        "metric": METRIC, "value": ms_per_frame, "unit": "ms/frame", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_frame, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
        "config": {"workload": WORKLOAD, "scene_triangles": mesh.triangle_count, "width": WIDTH, "height": HEIGHT,
                   "gi_resolution": [params.gi_width, params.gi_height], "di_lights": params.di_light_count,
                   "grid_table_size": params.grid_table_size, "graph": bool(args.graph),
                   "l2": "inputs larger than L2 (BVH 126 MB + frame targets), no flush",
                   "parallelism": f"replicas x{world}"},
        "mrays_per_s": float(rays / (ms_per_frame * 1e-3) / 1e6),
        "rays_per_frame": {"primary_and_shadow_map": int(counts[:, 0].sum()), "gi_closest": int(counts[:, 1].sum()),
                           "visibility_any_hit": int(counts[:, 2].sum())},
        "depth_buffer_marches_per_frame": int(counts[:, 3].sum()),
        "truncated_rays_per_frame": int(counts[:, 7].sum()),
        "rel_mse_vs_fp64_reference": plain_error["mean"], "rel_mse_median": plain_error["median"],
        "bias_vs_fp64_reference": plain_error["bias"], "rel_mse_frames": ERROR_FRAMES,
        "reference_frames": REFERENCE_FRAMES, "reference_noise": reference,
        "radiance_cache": cache_line,
        "radiance_cache_only_gi": cache_only_line,
        # The metric's comparison: plain ms/frame over the cache-only form's, when the
        # latter's relMSE is within the plain method's (else null).
        "plain_over_cache_at_equal_rel_mse": (ms_per_frame / cache_only_line["ms_per_frame"]
                                              if cache_only_line and cache_only_line["rel_mse_vs_fp64_reference"]
                                              <= plain_error["mean"] else None),
        "pass_ms": {name: float(mean_pass[i]) for i, name in enumerate(passes)},
        "side_stream_passes": list(SIDE_STREAM_PASSES),
        "pass_share": share,
        "pass_algorithmic_gbs": {name: (float(pass_bytes[name] / (mean_pass[i] * 1e-3) / 1e9) if mean_pass[i] > 0 else 0.0)
                                 for i, name in enumerate(passes)},
        "work_counts": {"node_fetches": int(counts[:, 4].sum()), "triangle_tests": int(counts[:, 5].sum()),
                        "depth_buffer_steps": int(counts[:, 6].sum())},
        "scene_setup_ms": scene_ms,
        "e2e": {"value": e2e_ms, "unit": "ms/frame", "h2d_bytes_per_step": 28, "d2h_bytes_per_step": 32,
                "api": "restir_renderer_render + restir_renderer_measure (error record read back) per step"},
        "gpu_launches": launches * args.steps,
        "roofline": {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": DOMINANT_TRAFFIC.get(name),
                     "traffic_source": "ncu DRAM read + write of the pass's kernels on this workload, one launch each",
                     "algorithmic_bytes_per_launch": footprint,
                     "algorithmic_bytes": "compulsory: the pass's image reads and writes plus each BVH row it "
                                          "touches at most once",
                     "fetched": {"bytes_per_launch": fetched_bytes[name], "achieved": fetched_gbs,
                                 "peak": l2_gather_gbs, "frac": fetched_gbs / l2_gather_gbs, "unit": "GB/s",
                                 "peak_source": "restir_gather_probe: random 32-byte gathers from the scene's BVH "
                                                "nodes (L2-resident), measured in this run"},
                     "limiter": "instruction issue and SIMT efficiency of divergent traversal (ncu: 9.3 of 32 "
                                "lanes active per instruction in the queue tracer, 66% of issue slots busy), "
                                "not DRAM bandwidth"},
        "cpu_baseline": baseline,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    renderer.close()
    if dist is not None:
        dist.destroy_process_group()


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=100)
    parser.add_argument("--warmup", type=int, default=5)
    parser.add_argument("--impl", default="own", choices=["own", "reference"])
    parser.add_argument("--graph", action="store_true", help="replay each frame as a CUDA graph")
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--no-cache", action="store_true", help="skip the radiance-cache form's measurement")
    parser.add_argument("--config", choices=["mid", "stress"], default=None,
                        help="another configuration of the metric's family (mid: 720p courtyard on a camera path; "
                             "stress: 4K, 4M triangles, 1,024 orbiting lights)")
    parser.add_argument("--batched", action="store_true",
                        help="the batched multi-view form (8 views of uneven resolution in one frame)")
    parser.add_argument("--cache-kernels", action="store_true",
                        help="time the radiance cache's query and training kernels alone (profiling)")
    parser.add_argument("--radiance-cache", action="store_true", help="with --quick: the radiance-cache form")
    parser.add_argument("--set", action="append", default=[], metavar="NAME=VALUE",
                        help="with --quick: a RestirSettings field (repeatable), e.g. --set cache_only_gi=1")
    parser.add_argument("--pareto", action="store_true",
                        help="both forms over several quality settings: ms/frame and relMSE, best at equal error")
    parser.add_argument("--bvh-build", action="store_true",
                        help="time the device BVH builder against the host builder (1M and 4M triangles)")
    parser.add_argument("--small", action="store_true",
                        help="with --quick: a smaller case of the frame for single-kernel ncu captures (the 1920x1080 "
                             "frame of the 100k-triangle city: its targets still exceed the L2, under 1 GB in all)")
    parser.add_argument("--quick", action="store_true",
                        help="profiling runs: W + K frames of the workload, no reference, no report")
    args = parser.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus if args.gpus == 1 else 1)))
    if args.cache_kernels:
        cache_kernels(args)
    elif args.bvh_build:
        bvh_build(args)
    elif args.pareto:
        pareto(args)
    elif args.config == "mid":
        mid_config(args)
    elif args.config == "stress":
        stress_config(args)
    elif args.batched:
        batched(args)
    elif args.impl == "reference":
        reference_arm(args, rank, world)
    else:
        own_arm(args, rank, world)


if __name__ == "__main__":
    main()
