"""The display kernels (restir_exposure, restir_taa, restir_tonemap and the
fused restir_display) against the oracle, bit for bit, on seeded images of
ragged sizes with background pixels, infinities, a NaN and half-range
extremes."""
import ctypes as C

import numpy as np
import pytest

import oracle.binding as ob
import restir_b200 as rb
from helpers import display_inputs, display_params

pytestmark = pytest.mark.gpu

SIZES = [(97, 61), (16, 8), (1, 1), (333, 7)]


def device(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def reference_planes(w, h, seed):
    rng = np.random.default_rng(seed)
    n = w * h
    return rng.lognormal(-1.0, 1.0, 3 * n), (rng.random(n) > 0.2).astype(np.uint8)


def oracle_display(p, inputs, exposure, mean, alpha):
    lib = ob.load()
    taa = np.zeros_like(inputs["hdr"])
    exposure = exposure.copy()
    if p.auto_exposure > 0.5 and p.pass_through <= 0.5:
        lib.oracle_exposure(C.byref(p), inputs["hdr"].ctypes.data, exposure.ctypes.data)
    image = inputs["hdr"]
    if p.taa > 0.5:
        lib.oracle_taa(C.byref(p), inputs["hdr"].ctypes.data, inputs["depth"].ctypes.data,
                       inputs["history"].ctypes.data, taa.ctypes.data)
        image = taa
    display = np.zeros(p.width * p.height * 4, np.uint8)
    lib.oracle_tonemap(C.byref(p), image.ctypes.data, exposure.ctypes.data, mean.ctypes.data, alpha.ctypes.data,
                       display.ctypes.data)
    return taa, exposure, display


@pytest.mark.parametrize("size", SIZES)
@pytest.mark.parametrize("valid,bottom_left", [(1.0, 0.0), (0.0, 0.0), (1.0, 1.0)])
def test_taa_bit_exact(size, valid, bottom_left):
    w, h = size
    inputs = display_inputs(w, h, seed=w * 7 + h)
    p = display_params(w, h, inputs, taa_history_valid=valid, origin_bottom_left=bottom_left)
    expected = np.zeros_like(inputs["hdr"])
    ob.load().oracle_taa(C.byref(p), inputs["hdr"].ctypes.data, inputs["depth"].ctypes.data,
                         inputs["history"].ctypes.data, expected.ctypes.data)
    d = {k: device(inputs[k]) for k in ("hdr", "depth", "history")}
    out = device(np.zeros_like(inputs["hdr"]))
    lib = rb.load()
    rb.check(lib.restir_taa(C.byref(p), d["hdr"].data_ptr(), d["depth"].data_ptr(), d["history"].data_ptr(),
                            out.data_ptr(), None), "restir_taa")
    np.testing.assert_array_equal(host(out), expected)


@pytest.mark.parametrize("op", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("auto", [0.0, 1.0])
def test_tonemap_bit_exact(op, auto):
    w, h = 97, 61
    inputs = display_inputs(w, h, seed=op + 10)
    exposure = np.array([np.float32(-1.75).view(np.uint32)], np.uint32)
    p = display_params(w, h, inputs, tonemapper=float(op), auto_exposure=auto, exposure_ev=0.75)
    expected = np.zeros(w * h * 4, np.uint8)
    ob.load().oracle_tonemap(C.byref(p), inputs["hdr"].ctypes.data, exposure.ctypes.data, None, None,
                             expected.ctypes.data)
    hdr, exp_d = device(inputs["hdr"]), device(exposure)
    out = device(np.zeros(w * h * 4, np.uint8))
    rb.check(rb.load().restir_tonemap(C.byref(p), hdr.data_ptr(), exp_d.data_ptr(), None, None, out.data_ptr(), None),
             "restir_tonemap")
    np.testing.assert_array_equal(host(out), expected)


@pytest.mark.parametrize("view,through", [(1.0, 0.0), (2.0, 0.0), (0.0, 1.0), (1.0, 1.0)])
def test_tonemap_reference_views_bit_exact(view, through):
    w, h = 61, 37
    inputs = display_inputs(w, h, seed=21)
    mean, alpha = reference_planes(w, h, 22)
    p = display_params(w, h, inputs, reference_view=view, pass_through=through)
    expected = np.zeros(w * h * 4, np.uint8)
    ob.load().oracle_tonemap(C.byref(p), inputs["hdr"].ctypes.data, None, mean.ctypes.data, alpha.ctypes.data,
                             expected.ctypes.data)
    hdr, mean_d, alpha_d = device(inputs["hdr"]), device(mean), device(alpha)
    out = device(np.zeros(w * h * 4, np.uint8))
    rb.check(rb.load().restir_tonemap(C.byref(p), hdr.data_ptr(), None, mean_d.data_ptr(), alpha_d.data_ptr(),
                                      out.data_ptr(), None), "restir_tonemap")
    np.testing.assert_array_equal(host(out), expected)


@pytest.mark.parametrize("size", [(97, 61), (1920, 1080), (7, 3)])
def test_exposure_bit_exact_over_frames(size):
    w, h = size
    lib, olib = rb.load(), ob.load()
    state = np.array([0], np.uint32)
    state_d = device(state)
    for frame in range(4):
        inputs = display_inputs(w, h, seed=frame + 30, specials=frame == 2)
        p = display_params(w, h, inputs, exposure_reset=1.0 if frame == 0 else 0.0, exposure_adapt=0.3)
        olib.oracle_exposure(C.byref(p), inputs["hdr"].ctypes.data, state.ctypes.data)
        hdr = device(inputs["hdr"])
        rb.check(lib.restir_exposure(C.byref(p), hdr.data_ptr(), state_d.data_ptr(), None), "restir_exposure")
        np.testing.assert_array_equal(host(state_d), state)
    assert abs(float(state.view(np.float32)[0])) < 12.0


@pytest.mark.parametrize("taa,auto,op", [(1.0, 1.0, 1), (1.0, 0.0, 0), (0.0, 1.0, 2), (1.0, 1.0, 3)])
def test_fused_display_equals_oracle_chain(taa, auto, op):
    w, h = 257, 129
    inputs = display_inputs(w, h, seed=40 + op)
    mean, alpha = reference_planes(w, h, 41)
    exposure = np.array([np.float32(0.5).view(np.uint32)], np.uint32)
    p = display_params(w, h, inputs, taa=taa, auto_exposure=auto, tonemapper=float(op), exposure_adapt=0.2)
    taa_expected, exposure_expected, display_expected = oracle_display(p, inputs, exposure, mean, alpha)
    d = {k: device(inputs[k]) for k in ("hdr", "depth", "history")}
    taa_out = device(np.zeros_like(inputs["hdr"]))
    exp_d, mean_d, alpha_d = device(exposure), device(mean), device(alpha)
    display = device(np.zeros(w * h * 4, np.uint8))
    rb.check(rb.load().restir_display(C.byref(p), d["hdr"].data_ptr(), d["depth"].data_ptr(), d["history"].data_ptr(),
                                      taa_out.data_ptr(), exp_d.data_ptr(), mean_d.data_ptr(), alpha_d.data_ptr(),
                                      display.data_ptr(), None), "restir_display")
    np.testing.assert_array_equal(host(display), display_expected)
    np.testing.assert_array_equal(host(exp_d), exposure_expected)
    if taa > 0.5:
        np.testing.assert_array_equal(host(taa_out), taa_expected)


def test_display_rejects_bad_arguments():
    lib = rb.load()
    w, h = 8, 8
    inputs = display_inputs(w, h, seed=50)
    p = display_params(w, h, inputs, auto_exposure=1.0)
    hdr = device(inputs["hdr"])
    out = device(np.zeros(w * h * 4, np.uint8))
    # auto exposure without the exposure word
    assert lib.restir_tonemap(C.byref(p), hdr.data_ptr(), None, None, None, out.data_ptr(), None) \
        == rb.ERROR_INVALID_ARGUMENT
    # TAA in place
    assert lib.restir_taa(C.byref(p), hdr.data_ptr(), hdr.data_ptr(), hdr.data_ptr(), hdr.data_ptr(), None) \
        == rb.ERROR_INVALID_ARGUMENT
    p.width = 0
    assert lib.restir_exposure(C.byref(p), hdr.data_ptr(), out.data_ptr(), None) == rb.ERROR_INVALID_ARGUMENT


def test_renderer_display_chain_equals_pass_by_pass_frames():
    """The frame driver's fused display launch and TAA ping-pong against the
    same frames run pass by pass (FrameRunner, separate exposure, TAA and
    tone-mapping calls), with auto exposure on."""
    from oracle.frame import FrameRunner
    from helpers import make_scene
    setup = make_scene(rb.SCENE_CORNELL)
    settings = setup.settings
    settings.gi_divisor = 1
    settings.grid_mode = rb.GRID_DETERMINISTIC
    settings.auto_exposure = 1
    w, h = 72, 40
    runner = FrameRunner(setup, w, h, "cuda", settings)
    renderer = rb.Renderer(settings)
    renderer.set_scene(setup.mesh, use_scene_defaults=False)
    frame = rb.frame_input(setup.mesh, w, h)
    for _ in range(4):
        runner.render()
        renderer.render(frame)
    _, plan, state = renderer.last_frame()
    assert plan.taa and plan.exposure and state.taa_valid and state.exposure_valid
    image = renderer.display_image()
    bgra = runner.host("display").reshape(h, w, 4)
    np.testing.assert_array_equal(image, bgra[..., [2, 1, 0, 3]])
    np.testing.assert_array_equal(renderer.download("display.hdr", np.uint16)[:w * h * 4],
                                  runner.host(runner.displayed()))
    np.testing.assert_array_equal(renderer.download("exposure", np.uint32)[:1], runner.host("exposure"))
