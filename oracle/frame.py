"""ORACLE (test infrastructure): the reference's per-frame pass sequence
(src/renderer.cpp:435-1125) over either backend, for parity tests and the
CPU baseline.

FrameRunner owns one frame's buffers and history with the reference's
ping-pong (renderer.h:218-219, renderer.cpp:706, 1122) and runs the passes in
the reference's order. backend="oracle" calls oracle/liboracle.so on numpy
arrays; backend="cuda" calls restir_b200's C ABI on torch tensors on cuda:0;
backend="ref" calls the reference's own shader code compiled as C++
(oracle/_ref/libref_shaders.so) for the passes it has (REF_PASSES) and the
oracle for the rest.
In check mode (run_checked) every CUDA pass is fed the oracle's inputs and
its outputs are compared with the oracle's bit for bit, pass by pass.

The frame uniforms come from the setup's host side: the library's own host
code (restir_frame_params) for tests.helpers.SceneSetup, the oracle's
restatement (oracle_frame_params) for oracle.workload.OracleSetup, which
needs nothing of the product's library.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

import restir_b200 as rb
from restir_b200.abi import RestirDiReservoirs, RestirGBuffer, RestirGiHistory, RestirGiReservoirs

from . import binding as ob

# Passes the reference's compiled shader code runs (backend "ref"): the
# compute and fragment passes of the light transport. The ray-cast stand-ins
# for the raster passes (G-buffer, shadow atlas), the FP64 reference and the
# display chain stay with the oracle.
REF_PASSES = ("grid_insert", "gi_temporal", "gi_spatial", "di_temporal", "di_spatial", "svgf_variance",
              "svgf_atrous", "composite_specular", "gi_specular")

# name: (dtype, channels, resolution) with resolution "full", "gi", "atlas", "grid", "none"
LAYOUT = {
    "gb.albedo": (np.uint8, 4, "full"), "gb.normal": (np.uint8, 4, "full"), "gb.emissive": (np.uint16, 4, "full"),
    "gb.shading_normal": (np.uint8, 4, "full"), "gb.depth": (np.float32, 1, "full"),
    "atlas": (np.float32, 1, "atlas"),
    "di.sample0": (np.float32, 4, "full"), "di.receiver0": (np.float32, 4, "full"), "di.normal0": (np.uint16, 4, "full"),
    "di.sample1": (np.float32, 4, "full"), "di.receiver1": (np.float32, 4, "full"), "di.normal1": (np.uint16, 4, "full"),
    "di.diffuse": (np.uint16, 4, "full"), "di.specular": (np.uint16, 4, "full"), "black": (np.uint16, 4, "full"),
    "grid0": (np.uint32, 1, "grid"), "grid1": (np.uint32, 1, "grid"),
    "gi.sample0": (np.float32, 4, "gi"), "gi.receiver0": (np.float32, 4, "gi"), "gi.normal0": (np.float32, 4, "gi"),
    "gi.sample1": (np.float32, 4, "gi"), "gi.receiver1": (np.float32, 4, "gi"), "gi.normal1": (np.float32, 4, "gi"),
    "gi.color0": (np.uint16, 4, "gi"), "gi.color1": (np.uint16, 4, "gi"),
    "gi.moments0": (np.uint16, 4, "gi"), "gi.moments1": (np.uint16, 4, "gi"),
    "filtered0": (np.uint16, 4, "gi"), "filtered1": (np.uint16, 4, "gi"),
    "filter0": (np.uint16, 4, "gi"), "filter1": (np.uint16, 4, "gi"),
    "hdr": (np.uint16, 4, "full"),
    "ref.mean": (np.float64, 3, "full"), "ref.alpha": (np.uint8, 1, "full"),
    "taa0": (np.uint16, 4, "full"), "taa1": (np.uint16, 4, "full"), "display": (np.uint8, 4, "full"),
    "specular0": (np.uint16, 4, "gi"), "specular1": (np.uint16, 4, "gi"),
    "exposure": (np.uint32, 1, "one"),
}


class ProductHost:
    """The host side of a frame through the product's library (restir_frame.h)."""

    def frame_params(self, settings, mesh, light_count, bvh, frame_input, state):
        return rb.frame_params(settings, mesh, light_count, bvh, frame_input, state)

    def advance(self, params, plan, frame_input, state):
        rb.advance(params, plan, frame_input, state)

    def display_params(self, *args):
        from restir_b200.abi import RestirDisplayParams
        out = RestirDisplayParams()
        rb.check(rb.load().restir_display_params(*args, C.byref(out)), "display_params")
        return out


class FrameRunner:
    def __init__(self, setup, width: int, height: int, backend: str = "oracle", settings=None,
                 gi_wavefront: bool = False):
        self.setup = setup
        self.backend = backend
        # cuda backend: the GI temporal and specular passes through their
        # wavefront forms (restir_gi_temporal_wavefront, restir_gi_specular_wavefront)
        self.gi_wavefront = gi_wavefront and backend == "cuda"
        self.gi_workspace = None
        self.specular_workspace = None
        self.settings = settings or setup.settings
        self.width, self.height = width, height
        self.state = rb.initial_state()
        self.history_read = 0
        self.di_read = 0
        self.taa_read = 0
        self.specular_read = 0
        self.display_taa = False
        self.params = None
        self.plan = None
        self.host_side = getattr(setup, "host_side", None) or ProductHost()
        self.frame_input = rb.frame_input(setup.mesh, width, height)
        p, _ = self.host_side.frame_params(self.settings, setup.mesh, setup.lights.count, setup.bvh, self.frame_input,
                                      self.state)
        self.shape = {"full": width * height, "gi": p.gi_width * p.gi_height,
                      "atlas": 6 * p.shadow_face_size * p.shadow_face_size,
                      "grid": p.grid_table_size * (2 + p.grid_cell_capacity), "one": 1}
        self.buffers = {}
        for name, (dt, ch, res) in LAYOUT.items():
            n = self.shape[res] * ch
            self.buffers[name] = np.zeros(n, dt)
        if backend == "cuda":
            import torch
            self.buffers = {k: torch.from_numpy(v).cuda() for k, v in self.buffers.items()}
            self.scene = setup.device_scene()
            self.lib = rb.load()
        else:
            self.scene = setup.host_scene()
            self.lib = ob.load()
            self.shader_lib = ob.load_shaders() if backend == "ref" else None
        self.error_scratch = None
        # The radiance cache (settings.radiance_cache): the cuda backend owns it;
        # the oracle backend takes its values per pass (cache_values) from there.
        self.radiance_cache = p.radiance_cache > 0.5
        self.cache = None
        self.cache_values = None
        if self.radiance_cache and backend == "cuda":
            desc = setup.mesh.desc
            lo = [desc.bounds_min[i] - 0.01 * desc.radius for i in range(3)]
            hi = [desc.bounds_max[i] + 0.01 * desc.radius for i in range(3)]
            self.cache = rb.RadianceCache(rb.cache_config(bounds_min=lo, bounds_max=hi))
            self.gi_wavefront = True

    # --- pass plumbing --------------------------------------------------------------------------------

    def b(self, name):
        return rb.ptr(self.buffers[name])

    def gbuffer(self) -> RestirGBuffer:
        g = RestirGBuffer()
        for f in ("albedo", "normal", "emissive", "shading_normal", "depth"):
            setattr(g, f, self.b("gb." + f))
        return g

    def call(self, name, *args):
        if self.backend == "cuda":
            rb.check(getattr(self.lib, "restir_" + name)(*args, None), name)
        elif self.backend == "ref" and name in REF_PASSES:
            rb.check(getattr(self.shader_lib, "ref_" + name)(*args), "ref_" + name)
        else:
            rb.check(getattr(self.lib, "oracle_" + name)(*args), name)

    def prepare(self):
        self.params, self.plan = self.host_side.frame_params(self.settings, self.setup.mesh, self.setup.lights.count,
                                                        self.setup.bvh, self.frame_input, self.state)
        return self.params, self.plan

    # --- the frame ------------------------------------------------------------------------------------

    def passes(self):
        """The frame as (pass name, callable) in the reference's order."""
        P, plan = self.params, self.plan
        hw = 1 - self.history_read
        hr = self.history_read
        dw = 1 - self.di_read
        gb = self.gbuffer()
        out = []
        out.append(("shadow_atlas", lambda: self.call("shadow_atlas", P, self.scene, self.b("atlas"))))
        out.append(("gbuffer_primary", lambda: self.call("gbuffer_primary", P, self.scene, gb)))
        if plan.di_active:
            prev = RestirDiReservoirs(self.b(f"di.sample{self.di_read}"), self.b(f"di.receiver{self.di_read}"),
                                      self.b(f"di.normal{self.di_read}"))
            cur = RestirDiReservoirs(self.b(f"di.sample{dw}"), self.b(f"di.receiver{dw}"), self.b(f"di.normal{dw}"))
            out.append(("di_temporal", lambda: self.call("di_temporal", P, self.scene, gb, prev, cur)))
            out.append(("di_spatial", lambda: self.call("di_spatial", P, self.scene, gb, cur, self.b("di.diffuse"),
                                                       self.b("di.specular"))))
        if plan.surface_light_is_di:
            surface = self.b("di.diffuse") if plan.di_active else self.b("black")
        else:
            surface = self.b("gb.emissive")
        out.append(("grid_clear", lambda: self.call("grid_clear", P, self.b(f"grid{hw}"))))
        out.append(("grid_insert", lambda: self.call("grid_insert", P, gb, self.b(f"grid{hw}"))))
        color_read = self.b(f"filtered{hr}") if plan.denoiser else self.b(f"gi.color{hr}")
        history = RestirGiHistory(self.b(f"gi.sample{hr}"), self.b(f"gi.receiver{hr}"), self.b(f"gi.normal{hr}"),
                                  color_read, self.b(f"gi.moments{hr}"))
        current = RestirGiReservoirs(self.b(f"gi.sample{hw}"), self.b(f"gi.receiver{hw}"), self.b(f"gi.normal{hw}"))
        if self.radiance_cache and self.backend == "cuda":
            out.append(("gi_temporal", lambda: self.cached_pass(
                "gi_temporal_cached", P, self.scene, gb, history, self.b(f"grid{hr}"), self.b("atlas"), surface,
                current)))
            out.append(("gi_spatial", lambda: self.cached_pass(
                "gi_spatial_cached", P, self.scene, gb, current, self.b(f"grid{hw}"), history, self.b("atlas"),
                surface, self.b(f"gi.color{hw}"), self.b(f"gi.moments{hw}"))))
            out.append(("cache_train", lambda: self.cached_pass("cache_train_frame", P, self.scene, gb,
                                                                self.b("atlas"))))
        elif self.radiance_cache:
            out.append(("gi_temporal", lambda: self.call(
                "gi_temporal_cached", P, self.scene, gb, history, self.b(f"grid{hr}"), self.b("atlas"), surface,
                current, self.cache_values.ctypes.data)))
            out.append(("gi_spatial", lambda: self.call(
                "gi_spatial_cached", P, self.scene, gb, current, self.b(f"grid{hw}"), history, self.b("atlas"),
                surface, self.b(f"gi.color{hw}"), self.b(f"gi.moments{hw}"), self.cache_values.ctypes.data)))
            out.append(("cache_train", lambda: None))
        else:
            if self.gi_wavefront:
                out.append(("gi_temporal", lambda: self.gi_temporal_wavefront(P, gb, history, self.b(f"grid{hr}"),
                                                                              surface, current)))
            else:
                out.append(("gi_temporal", lambda: self.call("gi_temporal", P, self.scene, gb, history,
                                                             self.b(f"grid{hr}"), self.b("atlas"), surface,
                                                             current)))
            out.append(("gi_spatial", lambda: self.call("gi_spatial", P, self.scene, gb, current,
                                                        self.b(f"grid{hw}"), history, self.b("atlas"), surface,
                                                        self.b(f"gi.color{hw}"), self.b(f"gi.moments{hw}"))))
        specular_write = f"specular{1 - self.specular_read}"
        if plan.specular and self.gi_wavefront:
            out.append(("gi_specular", lambda: self.gi_specular_wavefront(
                P, gb, history, surface, self.b(f"specular{self.specular_read}"), self.b(specular_write))))
        elif plan.specular:
            # Indirect specular (renderer.cpp:835-855): last frame's composite and specular history.
            out.append(("gi_specular", lambda: self.call(
                "gi_specular", P, self.scene, gb, history, self.b("atlas"), surface, self.b("hdr"),
                self.b(f"specular{self.specular_read}"), self.b(specular_write))))
        denoised = f"gi.color{hw}"
        if plan.denoiser:
            out.append(("svgf_variance", lambda: self.call("svgf_variance", P, self.b(f"gi.color{hw}"),
                                                           self.b(f"gi.moments{hw}"), self.b(f"gi.receiver{hw}"),
                                                           self.b(f"gi.normal{hw}"), self.b("filter0"))))
            for it in range(plan.atrous_iterations):
                src = "filter0" if it == 0 else (f"filtered{hw}" if it == 1 else f"filter{(it - 1) & 1}")
                dst = f"filtered{hw}" if it == 0 else f"filter{it & 1}"
                denoised = dst
                out.append((f"svgf_atrous{it}", (lambda s=src, d=dst, step=1 << it: self.call(
                    "svgf_atrous", P, step, self.b(s), self.b(f"gi.receiver{hw}"), self.b(f"gi.normal{hw}"),
                    self.b(d)))))
        di_d = self.b("di.diffuse") if plan.di_active else self.b("black")
        di_s = self.b("di.specular") if plan.di_active else self.b("black")
        spec = self.b(specular_write) if plan.specular else None
        out.append(("composite", lambda: self.call("composite_specular", P, gb, self.b("atlas"), self.b(denoised), di_d,
                                                   di_s, spec, self.b("hdr"))))
        if plan.reference_accumulate:
            out.append(("reference_accumulate", lambda: self.call(
                "reference_accumulate", P, self.b("hdr"), self.b("ref.mean"), self.b("ref.alpha"),
                plan.reference_weight_frames)))
        if plan.display:
            # Auto exposure, TAA and tone mapping (renderer.cpp:987-1117), as three passes.
            D = self.display_params()
            taa_read, taa_write = self.b(f"taa{self.taa_read}"), self.b(f"taa{1 - self.taa_read}")
            if plan.exposure:
                out.append(("exposure", lambda: self.call("exposure", C.byref(D), self.b("hdr"), self.b("exposure"))))
            if plan.taa:
                out.append(("taa", lambda: self.call("taa", C.byref(D), self.b("hdr"), self.b("gb.depth"), taa_read,
                                                     taa_write)))
            shown = taa_write if plan.taa else self.b("hdr")
            out.append(("tonemap", lambda: self.call("tonemap", C.byref(D), shown, self.b("exposure"), None, None,
                                                     self.b("display"))))
        return out

    def display_params(self):
        """The display passes' uniforms (restir_display_params or its restatement)."""
        P, plan, s = self.params, self.plan, self.settings
        inv = (C.c_float * 16)(*P.inv_view_proj)
        previous = (C.c_float * 16)(*self.state.previous_unjittered_view_proj)
        return self.host_side.display_params(C.cast(inv, C.c_void_p), C.cast(previous, C.c_void_p), P.width, P.height,
                                        plan.taa, self.state.taa_valid, plan.exposure, self.state.exposure_valid,
                                        s.adaptation_speed, self.frame_input.delta_time, s.exposure_ev, s.tonemapper,
                                        0, 0)

    def gi_temporal_wavefront(self, P, gb, history, grid, surface, current):
        import torch
        nbytes = int(self.lib.restir_gi_temporal_workspace_bytes(P))
        if self.gi_workspace is None or self.gi_workspace.numel() < nbytes:
            self.gi_workspace = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        assert self.gi_workspace.data_ptr() % 256 == 0
        rb.check(self.lib.restir_gi_temporal_wavefront(P, self.scene, gb, history, grid, self.b("atlas"), surface,
                                                        current, self.gi_workspace.data_ptr(), nbytes, None),
                 "gi_temporal_wavefront")

    def gi_specular_wavefront(self, P, gb, history, surface, specular_read, specular_write):
        import torch
        nbytes = int(self.lib.restir_gi_specular_workspace_bytes(P))
        if self.specular_workspace is None or self.specular_workspace.numel() < nbytes:
            self.specular_workspace = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        assert self.specular_workspace.data_ptr() % 256 == 0
        rb.check(self.lib.restir_gi_specular_wavefront(P, self.scene, gb, history, self.b("atlas"), surface,
                                                        self.b("hdr"), specular_read, specular_write,
                                                        self.specular_workspace.data_ptr(), nbytes, None),
                 "gi_specular_wavefront")

    def workspace(self, P):
        import torch
        nbytes = int(self.lib.restir_gi_temporal_workspace_bytes(P))
        if self.gi_workspace is None or self.gi_workspace.numel() < nbytes:
            self.gi_workspace = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
        assert self.gi_workspace.data_ptr() % 256 == 0
        return self.gi_workspace.data_ptr(), nbytes

    def cached_pass(self, name, *args):
        """A cuda pass of the radiance-cache path: its arguments, then the cache
        config and state and the GI workspace."""
        import ctypes as C
        pointer, nbytes = self.workspace(args[0])
        rb.check(getattr(self.lib, "restir_" + name)(*args, C.byref(self.cache.cfg), self.cache.state.data_ptr(), pointer,
                                                     nbytes, None), name)

    def cache_value_rows(self, P):
        """Host copy of the cache values the last cached pass read (half4 rows,
        candidates then reservoirs), from the workspace layout of
        restir_gi_temporal_workspace_bytes."""
        n = P.gi_width * P.gi_height * max(P.initial_candidates, 0)
        rows = n + P.gi_width * P.gi_height
        up = lambda b: (b + 255) // 256 * 256
        offset = up(8) + up(32 * n) + up(4 * n) + up(4 * n) + up(16 * n) + up(4 * n) + up(64 * rows)
        return self.gi_workspace[offset:offset + 8 * rows].cpu().numpy().view(np.uint16).copy()

    def finish(self):
        self.host_side.advance(self.params, self.plan, self.frame_input, self.state)
        self.history_read = 1 - self.history_read
        self.display_taa = bool(self.plan.display and self.plan.taa)
        if self.plan.specular:
            self.specular_read = 1 - self.specular_read
        if self.display_taa:
            self.taa_read = 1 - self.taa_read
        if self.plan.di_active:
            self.di_read = 1 - self.di_read

    def render(self):
        self.prepare()
        for _, fn in self.passes():
            fn()
        if self.backend == "cuda":
            import torch
            torch.cuda.synchronize()
        self.finish()

    def set_reference_accumulation(self, accumulate: bool):
        """Renderer::setReferenceAccumulation (renderer.cpp:1128-1141)."""
        if bool(self.state.reference_accumulating) == accumulate:
            return
        self.state.reference_accumulating = int(accumulate)
        if accumulate:
            self.state.reference_frames = 0
        self.state.history_valid = 0
        self.state.taa_valid = 0

    def displayed(self) -> str:
        """The buffer the last frame displayed: its TAA output, or the composite."""
        return f"taa{self.taa_read}" if self.display_taa else "hdr"

    def error(self) -> np.ndarray:
        """cs_error.sc against the reference, FP64: relMSE, mean image, mean reference, count."""
        P = self.params
        out = np.zeros(4, np.float64)
        if self.backend == "cuda":
            import torch
            if self.error_scratch is None:
                nbytes = self.lib.restir_error_scratch_bytes(self.width, self.height)
                self.error_scratch = torch.zeros(nbytes // 8 + 1, dtype=torch.float64, device="cuda")
            d = torch.zeros(4, dtype=torch.float64, device="cuda")
            rb.check(self.lib.restir_error(P, self.b(self.displayed()), self.b("ref.mean"), self.b("ref.alpha"), d.data_ptr(),
                                           self.error_scratch.data_ptr(), None), "error")
            out[:] = d.cpu().numpy()
        else:
            rb.check(self.lib.oracle_error(P, self.b(self.displayed()), self.b("ref.mean"), self.b("ref.alpha"),
                                           out.ctypes.data), "error")
        return out

    def host(self, name) -> np.ndarray:
        v = self.buffers[name]
        return v.cpu().numpy() if hasattr(v, "cpu") else v


def run_pinned(setup, width: int, height: int, frames: int, settings=None):
    """Runs `frames` frames with the oracle and with the reference's own
    shader code, feeding each reference pass the oracle's inputs and
    comparing its outputs bit for bit. Returns ({pass: mismatching elements},
    {pass the reference's code ran: output elements it changed})."""
    oracle_run = FrameRunner(setup, width, height, "oracle", settings)
    ref_run = FrameRunner(setup, width, height, "ref", settings)
    report, pinned = {}, {}
    for frame in range(frames):
        oracle_run.prepare()
        ref_run.prepare()
        for (name, o_fn), (_, r_fn) in zip(oracle_run.passes(), ref_run.passes()):
            before = {k: v.copy() for k, v in oracle_run.buffers.items()}
            for k, v in before.items():
                ref_run.buffers[k][...] = v
            o_fn()
            r_fn()
            base = name.rstrip("0123456789")
            base = "composite_specular" if base == "composite" else base
            if base not in REF_PASSES:
                continue
            for k in before:
                want, got = oracle_run.buffers[k], ref_run.buffers[k]
                changed = int(np.count_nonzero(got.view(np.uint8) != before[k].view(np.uint8)))
                pinned[base] = pinned.get(base, 0) + changed
                bad = int(np.count_nonzero(got.view(np.uint8) != want.view(np.uint8)))
                if bad:
                    report[f"{frame}:{name}:{k}"] = bad
        oracle_run.finish()
        ref_run.finish()
    return report, pinned


def run_checked(setup, width: int, height: int, frames: int, settings=None, on_mismatch=None,
                reference_frames: int = 0, gi_wavefront: bool = False):
    """Runs `frames` frames on both backends, feeding each CUDA pass the oracle's
    inputs and comparing its outputs bit for bit. Returns {pass: mismatching elements}."""
    import torch
    oracle_run = FrameRunner(setup, width, height, "oracle", settings)
    cuda_run = FrameRunner(setup, width, height, "cuda", settings, gi_wavefront=gi_wavefront)
    assert oracle_run.radiance_cache == cuda_run.radiance_cache
    report = {}
    # Buffers whose device copy may differ from the oracle's: all at first,
    # then those the last pass changed (the CUDA pass wrote its own values).
    stale = set(oracle_run.buffers)
    for frame in range(frames):
        if reference_frames and frame == frames - reference_frames:
            oracle_run.set_reference_accumulation(True)
            cuda_run.set_reference_accumulation(True)
        oracle_run.prepare()
        cuda_run.prepare()
        for (name, o_fn), (_, c_fn) in zip(oracle_run.passes(), cuda_run.passes()):
            before = {k: v.copy() for k, v in oracle_run.buffers.items()}
            # The CUDA pass gets exactly the oracle's inputs.
            for k in stale:
                cuda_run.buffers[k].copy_(torch.from_numpy(before[k]))
            if cuda_run.radiance_cache and name in ("gi_temporal", "gi_spatial", "cache_train"):
                # The cache lives on the GPU: the CUDA pass runs first and the
                # oracle takes the cache values it read.
                c_fn()
                torch.cuda.synchronize()
                if name != "cache_train":
                    oracle_run.cache_values = cuda_run.cache_value_rows(cuda_run.params)
                o_fn()
            else:
                o_fn()
                c_fn()
                torch.cuda.synchronize()
            changed = [k for k in before if not np.array_equal(before[k], oracle_run.buffers[k])]
            stale = set(changed) | ({k for k in before if k.startswith("grid")} if name.startswith("grid") else set())
            for k in changed + [k for k in before if k not in changed and name.startswith("grid")]:
                got = cuda_run.host(k)
                want = oracle_run.buffers[k]
                if k.startswith("grid"):
                    continue  # compared cell by cell in test_grid_gpu
                bad = int(np.count_nonzero(got.view(np.uint8) != want.view(np.uint8)))
                if bad:
                    report[f"{frame}:{name}:{k}"] = bad
                    if on_mismatch:
                        on_mismatch(frame, name, k, got, want)
            # Continue from the oracle's state for the grid (its slot order is scheduling-dependent).
        oracle_run.finish()
        cuda_run.finish()
    return report, oracle_run, cuda_run
