"""Every pass of a frame on the GPU against the oracle, bit for bit, over
several frames so that the history-dependent paths (temporal reuse through
last frame's grid, bounce light from the history, DI temporal reuse, the
denoiser's history) run: each CUDA pass gets exactly the oracle's inputs and
must reproduce the oracle's outputs. The grid runs in its deterministic mode
(cells list their lowest pixel indices in order), which fixes the entries
the reuse taps pick."""
import numpy as np
import pytest

import restir_b200 as rb
from oracle.frame import FrameRunner, run_checked
from tests.helpers import grid_cells, make_scene

CASES = {
    # Cornell box, full-resolution GI, its point light and emissive panel (DI over 2 triangles).
    "cornell": dict(scene=(rb.SCENE_CORNELL, 0, 0), size=(96, 96), frames=3, overrides=dict(gi_divisor=1)),
    # Courtyard, half-resolution GI, sky, 64 extra point lights and 256 emissive triangles.
    "courtyard": dict(scene=(rb.SCENE_COURTYARD, 0, 100000), size=(192, 108), frames=3,
                      overrides=dict(extra_lights=64)),
    # Every ray through the BVH, 4 GI candidates.
    "bvh-rays": dict(scene=(rb.SCENE_CORNELL, 0, 0), size=(64, 64), frames=2,
                     overrides=dict(gi_divisor=1, ray_mode=rb.RAY_BVH, initial_candidates=4)),
    # The display chain with auto exposure and ACES (every other case runs TAA and AgX, the defaults).
    "display-auto": dict(scene=(rb.SCENE_CORNELL, 0, 0), size=(96, 96), frames=4,
                         overrides=dict(gi_divisor=1, auto_exposure=1, tonemapper=0)),
    # Depth buffer only, screen-space reuse, GI without DI, no denoiser.
    "screen-space": dict(scene=(rb.SCENE_COURTYARD, 0, 20000), size=(128, 72), frames=3,
                         overrides=dict(ray_mode=rb.RAY_SCREEN, world_space_reuse=0, direct_lighting=1, denoiser=0)),
}


def _case_setup(case):
    c = CASES[case]
    kind, seed, tris = c["scene"]
    setup = make_scene(kind, seed, tris, extra_lights=c["overrides"].get("extra_lights", 0))
    settings = setup.settings
    for k, v in c["overrides"].items():
        setattr(settings, k, v)
    settings.grid_mode = rb.GRID_DETERMINISTIC
    if "extra_lights" in c["overrides"]:
        setup.lights = rb.Lights(setup.bvh, setup.mesh, settings)
    return c, setup, settings


@pytest.mark.gpu
@pytest.mark.parametrize("case", list(CASES))
def test_frame_passes_bit_exact(case):
    c, setup, settings = _case_setup(case)
    w, h = c["size"]
    report, oracle_run, cuda_run = run_checked(setup, w, h, c["frames"], settings)
    assert report == {}, report
    # The frames did real work: light arrived through GI and the image is not empty.
    hdr = oracle_run.host("hdr").view(np.uint16).reshape(-1, 4)
    assert np.count_nonzero(hdr[:, :3]) > 0.2 * hdr[:, :3].size
    gi = oracle_run.host("gi.color1" if oracle_run.history_read == 1 else "gi.color0")
    assert np.count_nonzero(gi) > 0
    # The display chain ran: TAA blended a history, the image is tone-mapped.
    assert oracle_run.display_taa and oracle_run.state.taa_valid
    assert np.count_nonzero(oracle_run.host("display")) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("case", list(CASES))
def test_gi_temporal_wavefront_bit_exact(case):
    """The wavefront GI temporal pass (candidates, queued tracer, shading) and
    the wavefront specular pass (rays, queued stackless walk, shading)
    reproduce the oracle's outputs bit for bit, like the single-kernel passes."""
    c, setup, settings = _case_setup(case)
    w, h = c["size"]
    rb.status_flags()
    report, _, cuda_run = run_checked(setup, w, h, c["frames"], settings, gi_wavefront=True)
    assert report == {}, report
    assert cuda_run.gi_workspace is not None
    assert rb.status_flags() & 4 == 0  # no queue overflow


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["courtyard", "bvh-rays"])
def test_wave_visibility_bit_exact(case):
    """Visibility rays in warp lock step (traceBvhWave, the reference's Vulkan
    path) reproduce the per-lane stackless walk's frame, pass by pass, as long
    as no warp reaches the step cap (checked)."""
    c, setup, settings = _case_setup(case)
    settings.wave_visibility = 1
    w, h = c["size"]
    rb.status_flags()
    report, _, _ = run_checked(setup, w, h, c["frames"], settings)
    assert report == {}, report
    assert rb.status_flags() & 1 == 0


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["cornell", "courtyard", "bvh-rays"])
def test_gi_passes_with_radiance_cache_bit_exact(case):
    """With the radiance cache standing in for previousIndirect, the GI passes
    reproduce the oracle's outputs bit for bit given the same cache values
    (the oracle reads the values the CUDA pass's queries returned); the cache
    trains every frame on path suffixes."""
    c, setup, settings = _case_setup(case)
    settings.radiance_cache = 1
    settings.cache_training_samples = 4096
    w, h = c["size"]
    rb.status_flags()
    report, oracle_run, cuda_run = run_checked(setup, w, h, c["frames"] + 1, settings)
    assert report == {}, report
    s = cuda_run.cache.scalars()
    assert s.step == c["frames"] + 1 and s.samples == 4096 and s.skipped_steps == 0
    values = oracle_run.cache_values.reshape(-1, 4)
    live = values[:, 3] == 0x3C00  # half 1.0: rows that were queries
    assert live.sum() > 0.2 * len(values)
    assert rb.status_flags() & (4 | 8) == 0


@pytest.mark.gpu
def test_gi_temporal_wavefront_rejects_bad_workspace():
    import torch
    setup = make_scene(rb.SCENE_CORNELL)
    runner = FrameRunner(setup, 32, 32, "cuda", gi_wavefront=True)
    P, _ = runner.prepare()
    lib = runner.lib
    nbytes = int(lib.restir_gi_temporal_workspace_bytes(P))
    n = P.gi_width * P.gi_height * P.initial_candidates
    assert nbytes == 256 + sum((b * n + 255) // 256 * 256 for b in (32, 4, 4, 16, 4))
    space = torch.zeros(nbytes + 256, dtype=torch.uint8, device="cuda")
    from restir_b200.abi import RestirGiHistory, RestirGiReservoirs
    hist = RestirGiHistory(runner.b("gi.sample0"), runner.b("gi.receiver0"), runner.b("gi.normal0"),
                           runner.b("gi.color0"), runner.b("gi.moments0"))
    cur = RestirGiReservoirs(runner.b("gi.sample1"), runner.b("gi.receiver1"), runner.b("gi.normal1"))
    args = (P, runner.scene, runner.gbuffer(), hist, runner.b("grid0"), runner.b("atlas"), runner.b("gb.emissive"), cur)
    # Misaligned, too small, missing.
    assert lib.restir_gi_temporal_wavefront(*args, space.data_ptr() + 16, nbytes, None) == rb.ERROR_INVALID_ARGUMENT
    assert lib.restir_gi_temporal_wavefront(*args, space.data_ptr(), nbytes - 1, None) == rb.ERROR_INVALID_ARGUMENT
    assert lib.restir_gi_temporal_wavefront(*args, None, nbytes, None) == rb.ERROR_INVALID_ARGUMENT
    torch.cuda.synchronize()


@pytest.mark.gpu
def test_gi_specular_wavefront_rejects_bad_workspace():
    import torch
    setup = make_scene(rb.SCENE_CORNELL)
    runner = FrameRunner(setup, 32, 32, "cuda", gi_wavefront=True)
    P, _ = runner.prepare()
    lib = runner.lib
    nbytes = int(lib.restir_gi_specular_workspace_bytes(P))
    n = P.gi_width * P.gi_height
    assert nbytes == 256 + sum((b * n + 255) // 256 * 256 for b in (32, 4, 4, 16))
    space = torch.zeros(nbytes + 256, dtype=torch.uint8, device="cuda")
    from restir_b200.abi import RestirGiHistory
    hist = RestirGiHistory(runner.b("gi.sample0"), runner.b("gi.receiver0"), runner.b("gi.normal0"),
                           runner.b("gi.color0"), runner.b("gi.moments0"))
    args = (P, runner.scene, runner.gbuffer(), hist, runner.b("atlas"), runner.b("gb.emissive"), runner.b("hdr"),
            runner.b("specular0"), runner.b("specular1"))
    # Misaligned, too small, missing.
    assert lib.restir_gi_specular_wavefront(*args, space.data_ptr() + 16, nbytes, None) == rb.ERROR_INVALID_ARGUMENT
    assert lib.restir_gi_specular_wavefront(*args, space.data_ptr(), nbytes - 1, None) == rb.ERROR_INVALID_ARGUMENT
    assert lib.restir_gi_specular_wavefront(*args, None, nbytes, None) == rb.ERROR_INVALID_ARGUMENT
    assert lib.restir_gi_specular_wavefront(*args, space.data_ptr(), nbytes, None) == rb.OK
    torch.cuda.synchronize()


@pytest.mark.gpu
def test_renderer_wavefront_frames_equal_single_kernel_frames():
    """The renderer's wavefront passes (GI temporal and specular through ray
    queues) give the single-kernel frames bit for bit on a 100k-triangle
    scene with sky, over frames that carry history."""
    mesh = rb.Mesh.procedural(rb.SCENE_COURTYARD, 2, 100000)
    frames = {}
    for wavefront in (0, 1):
        settings = rb.default_settings(mesh)
        settings.wavefront = wavefront
        settings.grid_mode = rb.GRID_DETERMINISTIC
        renderer = rb.Renderer(settings)
        renderer.set_scene(mesh, use_scene_defaults=False)
        frame = rb.frame_input(mesh, 240, 136)
        for _ in range(3):
            renderer.render(frame)
        frames[wavefront] = {name: renderer.download(name, np.uint16)
                             for name in ("specular0", "specular1", "hdr", "display.hdr")}
    for name in frames[0]:
        np.testing.assert_array_equal(frames[0][name], frames[1][name], err_msg=name)
    assert np.count_nonzero(frames[1]["specular0"]) + np.count_nonzero(frames[1]["specular1"]) > 0


@pytest.mark.gpu
def test_renderer_graph_frames_equal_stream_frames():
    """Frames replayed as CUDA graphs (restir_renderer_render_graph), with the
    side streams of the shadow atlas and the specular pass forked and joined
    inside each capture, equal the stream-launched frames bit for bit."""
    mesh = rb.Mesh.procedural(rb.SCENE_COURTYARD, 2, 50000)
    frames = {}
    for graph in (False, True):
        settings = rb.default_settings(mesh)
        settings.grid_mode = rb.GRID_DETERMINISTIC
        renderer = rb.Renderer(settings)
        renderer.set_scene(mesh, use_scene_defaults=False)
        frame = rb.frame_input(mesh, 160, 96)
        for _ in range(3):
            renderer.render(frame, graph=graph)
        frames[graph] = {name: renderer.download(name, np.uint16)
                         for name in ("hdr", "display.hdr", "specular0", "specular1", "shadow.atlas")}
    for name in frames[False]:
        np.testing.assert_array_equal(frames[False][name], frames[True][name], err_msg=name)
    assert np.count_nonzero(frames[True]["hdr"]) > 0


@pytest.mark.gpu
def test_reference_accumulation_and_error_fp64():
    setup = make_scene(rb.SCENE_CORNELL)
    settings = setup.settings
    settings.gi_divisor = 1
    settings.grid_mode = rb.GRID_DETERMINISTIC
    report, oracle_run, cuda_run = run_checked(setup, 64, 64, 4, settings, reference_frames=3)
    assert report == {}, report
    mean = oracle_run.host("ref.mean")
    assert np.count_nonzero(mean) > 0
    # The error pass: same record within FP64 summation-order rounding.
    cuda_run.buffers["ref.mean"].copy_(__import__("torch").from_numpy(mean))
    cuda_run.buffers["ref.alpha"].copy_(__import__("torch").from_numpy(oracle_run.host("ref.alpha")))
    cuda_run.buffers["hdr"].copy_(__import__("torch").from_numpy(oracle_run.host("hdr")))
    want = oracle_run.error()
    got = cuda_run.error()
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=0)
    assert want[3] > 0


@pytest.mark.gpu
def test_bench_configuration_frames_bit_exact():
    """The frame the benchmark times (1920x1080, the seeded 1M-triangle city,
    64 extra point lights beside its emissive panels, the reference's default
    settings: half-resolution GI with 2 candidates, 2 temporal and 4 spatial
    taps, ReSTIR DI, specular GI, SVGF with 5 a-trous levels, TAA and AgX),
    through the renderer's wavefront passes, three frames with history, every
    pass bit for bit against the oracle given the oracle's inputs. The grid
    runs in its deterministic mode (the atomic mode keeps the first 32
    arrivals per cell, which depends on scheduling)."""
    setup = make_scene(rb.SCENE_CITY, 0, 1_000_000, extra_lights=64)
    settings = setup.settings
    settings.grid_mode = rb.GRID_DETERMINISTIC
    assert (settings.gi_divisor, settings.initial_candidates, settings.atrous_iterations) == (2, 2, 5)
    rb.status_flags()
    report, oracle_run, cuda_run = run_checked(setup, 1920, 1080, 3, settings, gi_wavefront=True)
    assert report == {}, report
    assert setup.lights.count == 320 and setup.bvh.desc.triangle_count > 990_000
    gi = oracle_run.host("gi.color1" if oracle_run.history_read == 1 else "gi.color0")
    assert np.count_nonzero(gi) > 0.2 * gi.size
    assert rb.status_flags() & (2 | 4) == 0  # no probe-cap or queue overflow


@pytest.mark.gpu
def test_small_configuration_sixteen_frames_bit_exact():
    """The small configuration as stated: the procedural open-front Cornell box
    at 256x256, full-resolution GI (d = 1) with 1 candidate per pixel, a
    2^16-slot hash grid, GI temporal and spatial reuse, 16 static frames,
    seed 0; every pass of every frame bit for bit against the oracle."""
    setup = make_scene(rb.SCENE_CORNELL, 0, 0)
    settings = setup.settings
    settings.gi_divisor = 1
    settings.initial_candidates = 1
    settings.grid_mode = rb.GRID_DETERMINISTIC
    assert settings.grid_table_size == 1 << 16 and settings.temporal_taps > 0 and settings.spatial_taps > 0
    report, oracle_run, _ = run_checked(setup, 256, 256, 16, settings, gi_wavefront=True)
    assert report == {}, report
    assert oracle_run.state.frame_number == 16


@pytest.mark.gpu
def test_orbiting_extra_lights_move_and_hold():
    """RestirSettings.extra_light_orbit: the extra point lights move on circles
    about the scene's vertical axis from frame to frame (their height, colour
    and the emitters stay), and hold still when delta_time is 0."""
    mesh = rb.Mesh.procedural(rb.SCENE_COURTYARD, 0, 20000)
    settings = rb.default_settings(mesh)
    settings.extra_lights = 64
    settings.extra_light_orbit = 2.0
    renderer = rb.Renderer(settings)
    renderer.set_scene(mesh, use_scene_defaults=False)
    moving = rb.frame_input(mesh, 96, 64, delta_time=0.1)
    held = rb.frame_input(mesh, 96, 64, delta_time=0.0)
    lists = []
    for frame in (moving, moving, held, held):
        renderer.render(frame)
        lists.append(renderer.download("lights", np.float32).reshape(-1, 16).copy())
    center = np.array(mesh.desc.center, np.float32)
    emitters = int(np.count_nonzero(lists[0][:, 3] == 0.0))
    a, b = lists[0][emitters:], lists[1][emitters:]
    assert len(a) == 64 and not np.array_equal(a[:, [0, 2]], b[:, [0, 2]])
    np.testing.assert_array_equal(a[:, 1], b[:, 1])
    np.testing.assert_array_equal(a[:, 4:], b[:, 4:])
    np.testing.assert_allclose(np.hypot(a[:, 0] - center[0], a[:, 2] - center[2]),
                               np.hypot(b[:, 0] - center[0], b[:, 2] - center[2]), rtol=1e-5)
    np.testing.assert_array_equal(lists[0][:emitters], lists[1][:emitters])
    np.testing.assert_array_equal(lists[2], lists[3])
    hdr = renderer.download("hdr", np.float16)[:96 * 64 * 4].astype(np.float32)
    assert np.isfinite(hdr).all()
    renderer.close()


@pytest.mark.gpu
def test_saved_state_replays_the_following_frames(tmp_path):
    """restir_renderer_save_state / load_state: a second renderer loaded with
    the state saved after frame 3 renders frames 4 and 5 bit for bit as the
    first renderer does (history, reservoirs, grids, TAA and specular
    histories, frame number)."""
    mesh = rb.Mesh.procedural(rb.SCENE_COURTYARD, 1, 20000)
    frame = rb.frame_input(mesh, 160, 96)

    def make():
        settings = rb.default_settings(mesh)
        settings.grid_mode = rb.GRID_DETERMINISTIC
        settings.extra_lights = 16
        r = rb.Renderer(settings)
        r.set_scene(mesh, use_scene_defaults=False)
        return r

    first = make()
    for _ in range(3):
        first.render(frame)
    path = tmp_path / "frame3.state"
    first.save_state(path)
    for _ in range(2):
        first.render(frame)
    second = make()
    second.render(frame)  # targets of the same size
    second.load_state(path)
    for _ in range(2):
        second.render(frame)
    for name in ("display.hdr", "hdr", "display", "gi.sample0", "gi.sample1"):
        np.testing.assert_array_equal(first.download(name, np.uint8), second.download(name, np.uint8), err_msg=name)
    # The grids cell by cell: which slot a cell's key claims when two keys
    # probe the same slots depends on the order the inserting warps run in.
    settings = first.settings
    for name in ("grid0", "grid1"):
        cells = [grid_cells(r.download(name, np.uint32), settings.grid_table_size, settings.grid_cell_capacity)
                 for r in (first, second)]
        assert cells[0].keys() == cells[1].keys(), name
        for key, (count, entries) in cells[0].items():
            assert cells[1][key][0] == count, (name, key)
            np.testing.assert_array_equal(cells[1][key][1], entries, err_msg=name)
    assert first.last_frame()[2].frame_number == second.last_frame()[2].frame_number == 5
    # A file for targets of another size is refused.
    third = make()
    third.render(rb.frame_input(mesh, 64, 64))
    with pytest.raises(RuntimeError):
        third.load_state(path)
    for r in (first, second, third):
        r.close()
