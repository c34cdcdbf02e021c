"""The radiance cache's host side and oracle, without a GPU: the state
layout, and the oracle's gradients pinned against an independent float64
numpy restatement of the same network, itself checked by finite differences.
"""
import ctypes as C

import numpy as np

import oracle.binding as ob
import restir_b200 as rb
from restir_b200 import abi


def bf16_round(x):
    """float32 -> bfloat16 (nearest even) -> float64."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def test_layout():
    cfg = rb.cache_config(table_log2=12)
    layout = rb.cache_layout(cfg)
    offsets = [getattr(layout, f) for f, _ in abi.RestirCacheLayout._fields_[:12]]
    assert offsets == sorted(offsets) and all(o % 256 == 0 for o in offsets)
    assert layout.bytes == rb.load().restir_cache_state_bytes(C.byref(cfg))
    scales = list(layout.level_scale)
    assert scales[0] == 16.0 and scales[-1] == 2048.0 and scales == sorted(scales)
    assert all(float(s).is_integer() for s in scales)
    entries = 1 << 12
    for s, dense in zip(scales, layout.level_dense):
        assert bool(dense) == (8 * ((int(s) + 2) // 2) ** 3 <= entries)
    assert layout.table_half - layout.table == 16 * entries * 2 * 4
    bad = rb.cache_config(table_log2=30)
    assert rb.load().restir_cache_layout(C.byref(bad), C.byref(abi.RestirCacheLayout())) == rb.ERROR_INVALID_ARGUMENT


def numpy_network(w, x, targets, n, denom=None):
    """Forward and backward in float64 without rounding: loss, dL/dW and the
    loss's denominator (held constant in the gradient, so a finite difference
    must pass the unperturbed one back in)."""
    layers = [w[l * 4096:(l + 1) * 4096].reshape(64, 64) for l in range(4)] + [w[4 * 4096:].reshape(16, 64)]
    acts = [x]
    for l in range(4):
        acts.append(np.maximum(acts[-1] @ layers[l].T, 0.0))
    y = acts[-1] @ layers[4].T
    if denom is None:
        denom = y[:, :3] ** 2 + 0.01
    diff = y[:, :3] - targets[:, :3]
    loss = np.sum(diff ** 2 / denom) / (3 * n)
    dy = np.zeros_like(y)
    dy[:, :3] = 2.0 * diff / denom / (3 * n)
    grads = [None] * 5
    dz = dy
    for l in range(4, -1, -1):
        grads[l] = dz.T @ acts[l]
        dx = dz @ layers[l]
        if l > 0:
            dz = dx * (acts[l] > 0)
    return loss, np.concatenate([g.ravel() for g in grads]), denom


def test_oracle_gradients_against_numpy():
    rng = np.random.default_rng(0)
    n = 64
    w32 = np.zeros(abi.CACHE_WEIGHTS, np.float32)
    w32[:4 * 4096] = rng.uniform(-0.2, 0.2, 4 * 4096)
    w32[4 * 4096:4 * 4096 + 3 * 64] = rng.uniform(-0.3, 0.3, 3 * 64)
    w_bits = ((w32.view(np.uint32).astype(np.uint64) + 0x7FFF + ((w32.view(np.uint32) >> 16) & 1)) >> 16)
    w_bits = w_bits.astype(np.uint16)
    w = (w_bits.astype(np.uint32) << 16).view(np.float32).astype(np.float64)
    cfg = rb.cache_config(table_log2=12)
    layout = rb.cache_layout(cfg)
    table = np.zeros(16 * layout.entries * 2, np.uint16)  # zero features: inputs are the extra channels
    q = np.zeros((n, 16), np.float32)
    q[:, 0:3] = rng.uniform(0.0, 1.0, (n, 3))
    q[:, 3] = rng.uniform(0, 1, n)
    q[:, 4:7] = rng.normal(size=(n, 3))
    q[:, 8:11] = rng.normal(size=(n, 3))
    q[:, 12:15] = rng.uniform(0, 1, (n, 3))
    targets = rng.uniform(0.1, 1.0, (n, 4)).astype(np.float32)
    targets[:, 3] = 1.0
    feats = np.zeros((n, 64), np.uint16)
    lib = ob.load()
    lib.oracle_cache_features(C.byref(cfg), C.byref(layout), table.ctypes.data, q.ctypes.data, n, feats.ctypes.data)
    x = (feats.astype(np.uint32) << 16).view(np.float32).astype(np.float64)
    assert np.all(x[:, 42] == 1.0) and np.all(x[:, :32] == 0.0)
    np.testing.assert_array_equal(x[:, 32:35], bf16_round(q[:, 8:11]))

    want_loss, want, denom = numpy_network(w, x, targets.astype(np.float64), n)
    # Finite differences pin the numpy restatement's backward pass.
    for index in (5, 4096 + 77, 3 * 4096 + 1000, 4 * 4096 + 130):
        e = np.zeros_like(w)
        e[index] = 1e-6
        lp, _, _ = numpy_network(w + e, x, targets, n, denom)
        lm, _, _ = numpy_network(w - e, x, targets, n, denom)
        assert abs((lp - lm) / 2e-6 - want[index]) <= 1e-6 + 1e-4 * abs(want[index])

    got = np.zeros(abi.CACHE_WEIGHTS, np.float64)
    table_grad = np.zeros(table.size, np.float64)
    loss = C.c_double(0.0)
    lib.oracle_cache_gradients(C.byref(cfg), C.byref(layout), w_bits.ctypes.data, table.ctypes.data, q.ctypes.data,
                               targets.ctypes.data, n, C.c_float(128.0), got.ctypes.data, table_grad.ctypes.data,
                               C.byref(loss))
    assert abs(loss.value - want_loss) < 2e-2 * want_loss
    # The oracle rounds activations and layer gradients to bfloat16 as the
    # kernels do; against exact arithmetic that costs a few percent, most in
    # the layers furthest from the loss. A transposed or misindexed gradient
    # would be off by order one.
    for layer in range(5):
        lo, hi = layer * 4096, layer * 4096 + (4096 if layer < 4 else 3 * 64)
        err = np.linalg.norm(got[lo:hi] - want[lo:hi]) / np.linalg.norm(want[lo:hi])
        assert err < 0.1, (layer, err)


def test_oracle_adam_formula():
    cfg = rb.cache_config()
    rng = np.random.default_rng(1)
    n = 1000
    w = rng.normal(size=n).astype(np.float32)
    m = rng.normal(size=n).astype(np.float32) * 0.1
    v = np.abs(rng.normal(size=n)).astype(np.float32) * 0.01
    g = rng.normal(size=n).astype(np.float32)
    b1p, b2p = np.float32(0.9 ** 3), np.float32(0.99 ** 3)
    w2, m2, v2 = w.copy(), m.copy(), v.copy()
    ob.load().oracle_cache_adam(C.byref(cfg), n, w2.ctypes.data, m2.ctypes.data, v2.ctypes.data, g.ctypes.data,
                                C.c_float(b1p), C.c_float(b2p))
    f = np.float32
    b1, b2, lr, eps = f(cfg.beta1), f(cfg.beta2), f(cfg.learning_rate), f(cfg.epsilon)
    em = b1 * m + (f(1) - b1) * g
    ev = b2 * v + (f(1) - b2) * (g * g)
    ew = w - (lr * (em / (f(1) - b1p))) / (np.sqrt(ev / (f(1) - b2p)) + eps)
    np.testing.assert_array_equal(m2, em)
    np.testing.assert_array_equal(v2, ev)
    np.testing.assert_array_equal(w2, ew)
