"""The display passes' oracle (oracle/oracle_display.cpp) against a second,
independent restatement of fs_taa.sc, cs_exposure.sc and fs_tonemap.sc /
tonemap.sh in float64 numpy, and the host-side uniform derivation. The CUDA
kernels are checked bit for bit against the oracle in test_display_gpu.py."""
import ctypes as C
import math

import numpy as np
import pytest

import oracle.binding as ob
import restir_b200 as rb
from restir_b200.abi import RestirDisplayParams
from helpers import display_inputs, display_params

LUMINANCE = np.array([0.2126, 0.7152, 0.0722])


def halves(bits: np.ndarray, height: int, width: int) -> np.ndarray:
    return bits.view(np.float16).astype(np.float64).reshape(height, width, 4)


def oracle_taa(p, inputs):
    out = np.zeros_like(inputs["hdr"])
    ob.load().oracle_taa(C.byref(p), inputs["hdr"].ctypes.data, inputs["depth"].ctypes.data,
                         inputs["history"].ctypes.data, out.ctypes.data)
    return out


def oracle_tonemap(p, hdr, exposure=None, mean=None, alpha=None):
    display = np.zeros(p.width * p.height * 4, np.uint8)
    ob.load().oracle_tonemap(C.byref(p), hdr.ctypes.data, None if exposure is None else exposure.ctypes.data,
                             None if mean is None else mean.ctypes.data, None if alpha is None else alpha.ctypes.data,
                             display.ctypes.data)
    return display.reshape(p.height, p.width, 4)


# --- numpy float64 restatement ---------------------------------------------------------------------------------

def np_bilinear(img, u, v):
    h, w = img.shape[:2]
    px, py = u * w - 0.5, v * h - 0.5
    bx, by = math.floor(px), math.floor(py)
    fx, fy = px - bx, py - by
    x0, x1 = min(max(bx, 0), w - 1), min(max(bx + 1, 0), w - 1)
    y0, y1 = min(max(by, 0), h - 1), min(max(by + 1, 0), h - 1)
    top = img[y0, x0, :3] * (1 - fx) + img[y0, x1, :3] * fx
    bottom = img[y1, x0, :3] * (1 - fx) + img[y1, x1, :3] * fx
    return top * (1 - fy) + bottom * fy


def np_history(img, uv):
    h, w = img.shape[:2]
    texel = np.array([1.0 / w, 1.0 / h])
    position = uv / texel
    center = np.floor(position - 0.5) + 0.5
    f = position - center
    w0 = f * (-0.5 + f * (1.0 - 0.5 * f))
    w1 = 1.0 + f * f * (-2.5 + 1.5 * f)
    w2 = f * (0.5 + f * (2.0 - 1.5 * f))
    w3 = f * f * (-0.5 + 0.5 * f)
    w12 = w1 + w2
    o12 = w2 / w12
    uv0, uv3, uv12 = (center - 1.0) * texel, (center + 2.0) * texel, (center + o12) * texel
    taps = [((uv12[0], uv0[1]), w12[0] * w0[1]), ((uv0[0], uv12[1]), w0[0] * w12[1]),
            ((uv12[0], uv12[1]), w12[0] * w12[1]), ((uv3[0], uv12[1]), w3[0] * w12[1]),
            ((uv12[0], uv3[1]), w12[0] * w3[1])]
    color = sum(np_bilinear(img, u, v) * wt for (u, v), wt in taps)
    return np.maximum(color / sum(wt for _, wt in taps), 0.0)


def ycocg(c):
    return np.array([c @ [0.25, 0.5, 0.25], c @ [0.5, 0.0, -0.5], c @ [-0.25, 0.5, -0.25]])


def np_taa_pixel(hdr, depth, history, inv, previous, x, y, valid):
    h, w = hdr.shape[:2]
    texel = np.array([1.0 / w, 1.0 / h])
    uv = (np.array([x, y]) + 0.5) * texel
    current = hdr[y, x]
    stats, nearest, nearest_uv = [], 1.0, uv
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            tx, ty = min(max(x + dx, 0), w - 1), min(max(y + dy, 0), h - 1)
            c = hdr[ty, tx, :3]
            stats.append(ycocg(c / (1.0 + c @ LUMINANCE)))
            if depth[ty, tx] < nearest:
                nearest, nearest_uv = depth[ty, tx], uv + np.array([dx, dy]) * texel
    if not valid:
        return current
    clip = np.array([nearest_uv[0] * 2 - 1, -(nearest_uv[1] * 2 - 1), nearest, 1.0])
    world = inv @ clip
    world = np.append(world[:3] / world[3], 1.0)
    pc = previous @ world
    puv = np.array([pc[0] / pc[3], -pc[1] / pc[3]]) * 0.5 + 0.5 + (uv - nearest_uv)
    if pc[3] <= 1e-4 or np.any(puv < 0.0) or np.any(puv > 1.0):
        return current
    stats = np.array(stats)
    mean = stats.mean(axis=0)
    deviation = np.sqrt(np.maximum((stats ** 2).mean(axis=0) - mean ** 2, 0.0)) * 1.25
    past = np_history(history, puv)
    past = ycocg(past / (1.0 + past @ LUMINANCE))
    offset = past - mean
    largest = np.max(np.abs(offset / np.maximum(deviation, 1e-5)))
    if largest > 1.0:
        past = mean + offset / largest
    rgb = np.array([past[0] + past[1] - past[2], past[0] + past[2], past[0] - past[1] - past[2]])
    cur = current[:3] / (1.0 + current[:3] @ LUMINANCE)
    blended = rgb * 0.9 + cur * 0.1
    result = blended / max(1.0 - blended @ LUMINANCE, 1e-4)
    return np.append(result, current[3])


def np_aces(c):
    a_in = np.array([[0.59719, 0.35458, 0.04823], [0.07600, 0.90834, 0.01566], [0.02840, 0.13383, 0.83777]])
    a_out = np.array([[1.60475, -0.53108, -0.07367], [-0.10208, 1.10813, -0.00605], [-0.00327, -0.07276, 1.07602]])
    v = c @ a_in.T
    a = v * (v + 0.0245786) - 0.000090537
    b = v * (0.983729 * v + 0.4329510) + 0.238081
    return np.clip((a / b) @ a_out.T, 0.0, 1.0)


def np_agx(c):
    inset = np.array([[0.842479062253094, 0.0784335999999992, 0.0792237451477643],
                      [0.0423282422610123, 0.878468636469772, 0.0791661274605434],
                      [0.0423756549057051, 0.0784336, 0.879142973793104]])
    outset = np.array([[1.19687900512017, -0.0980208811401368, -0.0990297440797205],
                       [-0.0528968517574562, 1.15190312990417, -0.0989611768448433],
                       [-0.0529716355144438, -0.0980434501171241, 1.15107367264116]])
    lo, hi = -12.47393, 4.026069
    v = np.maximum(c, 0.0) @ inset.T
    v = (np.clip(np.log2(np.maximum(v, 1e-10)), lo, hi) - lo) / (hi - lo)
    x2, x4 = v * v, v ** 4
    v = 15.5 * x4 * x2 - 40.14 * x4 * v + 31.96 * x4 - 6.868 * x2 * v + 0.4298 * x2 + 0.1191 * v - 0.00232
    return np.clip(v @ outset.T, 0.0, 1.0) ** 2.2


def np_neutral(c):
    out = np.empty_like(c)
    for i, col in enumerate(c):
        x = col.min()
        col = col - (x - 6.25 * x * x if x < 0.08 else 0.04)
        peak = col.max()
        if peak < 0.76:
            out[i] = np.clip(col, 0, 1)
            continue
        d = 0.24
        new_peak = 1.0 - d * d / (peak + d - 0.76)
        col = col * new_peak / peak
        g = 1.0 - 1.0 / (0.15 * (peak - new_peak) + 1.0)
        out[i] = np.clip(col * (1 - g) + new_peak * g, 0, 1)
    return out


OPERATORS = {0: np_aces, 1: np_agx, 2: np_neutral, 3: lambda c: c / (c + 1.0), 4: lambda c: np.clip(c, 0.0, 1.0)}


def np_turbo(x):
    x = np.clip(x, 0.0, 1.0)
    v4 = np.stack([np.ones_like(x), x, x * x, x ** 3], axis=-1)
    v2 = np.stack([x ** 4, x ** 5], axis=-1)
    r = v4 @ [0.13572138, 4.61539260, -42.66032258, 132.13108234] + v2 @ [-152.94239396, 59.28637943]
    g = v4 @ [0.09140261, 2.19418839, 4.84296658, -14.18503333] + v2 @ [4.27729857, 2.82956604]
    b = v4 @ [0.10667330, 12.64194608, -60.58204836, 110.36276771] + v2 @ [-89.90310912, 27.34824973]
    return np.stack([r, g, b], axis=-1)


def to_bgra8(rgb):
    q = np.floor(np.clip(rgb, 0.0, 1.0) * 255.0 + 0.5).astype(np.int32)
    return q[..., [2, 1, 0]]


# --- tests ------------------------------------------------------------------------------------------------------

@pytest.mark.parametrize("valid", [False, True])
def test_oracle_taa_matches_float64_restatement(valid):
    w, h = 23, 17
    inputs = display_inputs(w, h, seed=3, specials=False)
    p = display_params(w, h, inputs, taa_history_valid=1.0 if valid else 0.0)
    out = halves(oracle_taa(p, inputs), h, w)
    hdr = halves(inputs["hdr"], h, w)
    history = halves(inputs["history"], h, w)
    depth = inputs["depth"].astype(np.float64).reshape(h, w)
    inv = inputs["inv_view_proj"].astype(np.float64)
    previous = inputs["previous_view_proj"].astype(np.float64)
    reprojected = 0
    close = 0
    for y in range(h):
        for x in range(w):
            expected = np_taa_pixel(hdr, depth, history, inv, previous, x, y, valid)
            reprojected += not np.array_equal(expected, hdr[y, x])
            close += np.allclose(out[y, x], expected, rtol=4e-3, atol=1e-4)
    if valid:
        assert reprojected > 0.8 * w * h
        assert close >= w * h - 2  # a clip decision at the edge of float32 may flip
    else:
        assert close == w * h
        np.testing.assert_array_equal(oracle_taa(p, inputs), inputs["hdr"])


def test_oracle_taa_nan_guard():
    w, h = 9, 7
    inputs = display_inputs(w, h, seed=4, specials=True)
    p = display_params(w, h, inputs)
    out = halves(oracle_taa(p, inputs), h, w)
    assert np.all(np.isfinite(out[..., :3]) | np.isinf(halves(inputs["hdr"], h, w)[..., :3]))
    assert not np.any(np.isnan(out))


@pytest.mark.parametrize("op", [0, 1, 2, 3, 4])
def test_oracle_tonemap_operators_match_float64(op):
    w, h = 31, 9
    inputs = display_inputs(w, h, seed=5, specials=False)
    p = display_params(w, h, inputs, tonemapper=float(op), exposure_ev=0.5)
    display = oracle_tonemap(p, inputs["hdr"]).astype(np.int32)
    hdr = halves(inputs["hdr"], h, w).reshape(-1, 4)
    color = OPERATORS[op](hdr[:, :3] * 2.0 ** 0.5)
    expected = to_bgra8(np.abs(color) ** (1.0 / 2.2))
    background = hdr[:, 3] < 0.5
    expected[background] = to_bgra8(np.array([0.125, 0.141, 0.169]))
    got = display.reshape(-1, 4)
    assert np.max(np.abs(got[:, :3] - expected)) <= 1
    assert np.all(got[:, 3] == 255)


def test_oracle_exposure_and_auto_tonemap():
    w, h = 200, 120
    inputs = display_inputs(w, h, seed=6, specials=False)
    hdr = halves(inputs["hdr"], h, w)
    logs = []
    for gy in range(64):
        for gx in range(64):
            tx = min(int(math.floor((gx + 0.5) / 64.0 * w)), w - 1)
            ty = min(int(math.floor((gy + 0.5) / 64.0 * h)), h - 1)
            if hdr[ty, tx, 3] > 0.5:
                logs.append(np.clip(np.log2(max(hdr[ty, tx, :3] @ LUMINANCE, 1e-6)), -12, 12))
    average = float(np.mean(logs))
    exposure = np.array([np.float32(100.0).view(np.uint32)], np.uint32)  # out of range: resets
    p = display_params(w, h, inputs, exposure_adapt=0.25)
    ob.load().oracle_exposure(C.byref(p), inputs["hdr"].ctypes.data, exposure.ctypes.data)
    first = float(exposure.view(np.float32)[0])
    assert abs(first - average) < 1e-4
    exposure[0] = np.float32(1.0).view(np.uint32)
    ob.load().oracle_exposure(C.byref(p), inputs["hdr"].ctypes.data, exposure.ctypes.data)
    assert abs(float(exposure.view(np.float32)[0]) - (0.75 * 1.0 + 0.25 * average)) < 1e-4
    # tone mapping with auto exposure: 2^EV * 0.18 / 2^adapted
    adapted = float(exposure.view(np.float32)[0])
    p = display_params(w, h, inputs, tonemapper=4.0, auto_exposure=1.0)
    got = oracle_tonemap(p, inputs["hdr"], exposure).astype(np.int32).reshape(-1, 4)
    flat = hdr.reshape(-1, 4)
    expected = to_bgra8(np.clip(flat[:, :3] * 0.18 / 2.0 ** adapted, 0, 1) ** (1 / 2.2))
    geometry = flat[:, 3] >= 0.5
    assert np.max(np.abs(got[geometry, :3] - expected[geometry])) <= 1
    # only background: the stored value stays
    empty = inputs["hdr"].copy().view(np.float16).reshape(-1, 4)
    empty[:, 3] = 0.0
    before = exposure.copy()
    ob.load().oracle_exposure(C.byref(p), empty.view(np.uint16).reshape(-1).ctypes.data, exposure.ctypes.data)
    assert exposure[0] == before[0]


def test_oracle_reference_views():
    w, h = 13, 11
    inputs = display_inputs(w, h, seed=7, specials=False)
    n = w * h
    rng = np.random.default_rng(8)
    mean = rng.lognormal(-1.0, 1.0, 3 * n)
    alpha = (rng.random(n) > 0.2).astype(np.uint8)
    hdr = halves(inputs["hdr"], h, w).reshape(-1, 4)
    p = display_params(w, h, inputs, reference_view=2.0)
    got = oracle_tonemap(p, inputs["hdr"], None, mean, alpha).astype(np.int32).reshape(-1, 4)
    ref = np.stack([mean[:n], mean[n:2 * n], mean[2 * n:]], axis=-1).astype(np.float32).astype(np.float64)
    error = (hdr[:, :3] @ LUMINANCE - ref @ LUMINANCE) / np.maximum(ref @ LUMINANCE, 0.01)
    expected = to_bgra8(np_turbo(0.5 + np.clip(error, -0.5, 0.5)))
    expected[alpha == 0] = to_bgra8(np.array([0.125, 0.141, 0.169]))
    assert np.max(np.abs(got[:, :3] - expected)) <= 1
    p = display_params(w, h, inputs, reference_view=1.0, pass_through=1.0)
    got = oracle_tonemap(p, inputs["hdr"], None, mean, alpha).astype(np.int32).reshape(-1, 4)
    assert np.max(np.abs(got[:, :3] - to_bgra8(ref))) <= 1


def test_display_params_follow_the_renderer():
    lib = rb.load()
    inv = np.arange(16, dtype=np.float32)
    prev = np.arange(16, 32, dtype=np.float32)
    p = RestirDisplayParams()
    assert lib.restir_display_params(inv.ctypes.data, prev.ctypes.data, 64, 32, 1, 1, 1, 0, 1.5, 1.0 / 60.0, -0.5,
                                     rb.abi.TONEMAP_AGX, 0, 0, C.byref(p)) == rb.OK
    assert list(p.inv_view_proj) == list(inv) and list(p.previous_view_proj) == list(prev)
    assert p.taa == 1.0 and p.taa_history_valid == 1.0 and p.exposure_reset == 1.0
    assert abs(p.exposure_adapt - (1.0 - math.exp(-1.5 / 60.0))) < 1e-7
    assert p.tonemapper == 1.0 and p.exposure_ev == -0.5 and p.auto_exposure == 1.0
    # a data view turns TAA off
    assert lib.restir_display_params(inv.ctypes.data, prev.ctypes.data, 64, 32, 1, 1, 0, 1, 1.5, 0.0, 0.0, 0, 1, 0,
                                     C.byref(p)) == rb.OK
    assert p.taa == 0.0 and p.pass_through == 1.0
    assert lib.restir_display_params(inv.ctypes.data, prev.ctypes.data, 64, 32, 1, 1, 0, 1, 1.5, 0.0, 0.0, 9, 0, 0,
                                     C.byref(p)) == rb.ERROR_INVALID_ARGUMENT
