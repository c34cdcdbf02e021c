"""The radiance cache's kernels (restir_cache_*) against the oracle's
restatement (oracle/oracle_cache.cpp): the hash-grid inputs bit for bit, the
tensor-core MLP's outputs and gradients to the tolerance bfloat16 operands
with FP32 accumulation allow, Adam bit for bit, and training that fits a
target."""
import ctypes as C

import numpy as np
import pytest

import oracle.binding as ob
import restir_b200 as rb
from restir_b200 import abi

N_SMALL = 1000


def make_queries(n, seed=0, lo=(-2.0, -1.0, -3.0), hi=(2.0, 3.0, 1.0)):
    rng = np.random.default_rng(seed)
    q = np.zeros((n, 16), np.float32)
    q[:, 0:3] = rng.uniform(lo, hi, (n, 3))
    q[:, 3] = rng.uniform(0.0, 1.0, n)
    for col in (4, 8):
        v = rng.normal(size=(n, 3))
        q[:, col:col + 3] = v / np.linalg.norm(v, axis=1, keepdims=True)
    q[:, 12:15] = rng.uniform(0.05, 0.95, (n, 3))
    q[:, 7] = 1.0  # valid
    return q


def target_function(q):
    """A smooth positive radiance over position and normal."""
    p = q[:, 0:3]
    t = np.zeros((len(q), 4), np.float32)
    t[:, 3] = 1.0  # weight
    t[:, 0] = 0.6 + 0.4 * np.sin(2.0 * p[:, 0]) * np.cos(1.5 * p[:, 1])
    t[:, 1] = 0.5 + 0.3 * q[:, 5] + 0.1 * np.sin(3.0 * p[:, 2])
    t[:, 2] = 0.3 + 0.2 * np.cos(p[:, 0] + p[:, 2])
    return t


def small_cache(**overrides):
    fields = dict(bounds_min=(-2.0, -1.0, -3.0), bounds_max=(2.0, 3.0, 1.0), table_log2=12)
    fields.update(overrides)
    return rb.RadianceCache(rb.cache_config(**fields))


def host_region(cache, name, dtype):
    return cache.region(name, dtype).cpu().numpy()


@pytest.fixture(scope="module")
def trained():
    """A cache after 50 training steps, so that the hash table is not tiny."""
    import torch
    cache = small_cache()
    q = make_queries(8192, seed=7)
    t = target_function(q)
    dq = torch.from_numpy(q).cuda()
    dt = torch.from_numpy(t).cuda()
    for _ in range(50):
        cache.train(dq, dt)
    torch.cuda.synchronize()
    return cache


@pytest.mark.gpu
def test_features_bit_exact(trained):
    import torch
    q = make_queries(N_SMALL, seed=1)
    got = trained.features(torch.from_numpy(q).cuda()).cpu().numpy().view(np.uint16)
    want = np.zeros((N_SMALL, 64), np.uint16)
    table = host_region(trained, "table_half", torch.int16).view(np.uint16)
    ob.load().oracle_cache_features(C.byref(trained.cfg), C.byref(trained.layout), table.ctypes.data, q.ctypes.data,
                                    N_SMALL, want.ctypes.data)
    np.testing.assert_array_equal(got, want)
    assert np.count_nonzero(want[:, :32]) > 0.9 * want[:, :32].size


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 127, 128, 1000, 5000])
def test_forward_matches_oracle(trained, n):
    import torch
    q = make_queries(n, seed=2)
    dq = torch.from_numpy(q).cuda()
    got = trained.forward(dq).cpu().numpy()
    inputs = trained.features(dq).cpu().numpy().view(np.uint16)
    weights = host_region(trained, "weights_bf16", torch.int16).view(np.uint16)
    want = np.zeros((n, 16), np.float64)
    ob.load().oracle_cache_forward(weights.ctypes.data, inputs.ctypes.data, n, want.ctypes.data)
    scale = np.abs(want[:, :3]).mean() + 1e-6
    np.testing.assert_allclose(got[:, :3], want[:, :3], rtol=2e-2, atol=2e-2 * scale)
    # The padding outputs have zero weights.
    assert np.all(got[:, 3:] == 0.0)
    # query() is max(output, 0) as half, alpha the query's valid flag.
    q[::2, 7] = 0.0
    h = trained.query(torch.from_numpy(q).cuda()).cpu().numpy().astype(np.float32)
    np.testing.assert_allclose(h[:, :3], np.maximum(got[:, :3], 0.0), rtol=1e-3, atol=1e-4)
    np.testing.assert_array_equal(h[:, 3], q[:, 7])


@pytest.mark.gpu
@pytest.mark.parametrize("n", [200, 4096])
def test_gradients_match_oracle(trained, n):
    import torch
    q = make_queries(n, seed=3)
    t = target_function(q)
    t[::3, 3] = 0.0  # samples of weight 0 drop out of the loss and the gradients
    weights = host_region(trained, "weights_bf16", torch.int16).view(np.uint16).copy()
    table = host_region(trained, "table_half", torch.int16).view(np.uint16).copy()
    scale = trained.scalars().loss_scale
    trained.gradients(torch.from_numpy(q).cuda(), torch.from_numpy(t).cuda())
    torch.cuda.synchronize()
    got_w = host_region(trained, "weight_grad", torch.float32)[:abi.CACHE_WEIGHTS]
    got_t = host_region(trained, "table_grad", torch.float32)
    want_w = np.zeros(abi.CACHE_WEIGHTS, np.float64)
    want_t = np.zeros(got_t.size, np.float64)
    loss = C.c_double(0.0)
    ob.load().oracle_cache_gradients(C.byref(trained.cfg), C.byref(trained.layout), weights.ctypes.data,
                                     table.ctypes.data, q.ctypes.data, t.ctypes.data, n, C.c_float(scale),
                                     want_w.ctypes.data, want_t.ctypes.data, C.byref(loss))
    s = trained.scalars()
    assert s.nonfinite == 0 and s.samples == n
    assert s.loss == pytest.approx(loss.value, rel=2e-2)
    for layer in range(5):
        lo, hi = layer * 4096, layer * 4096 + (4096 if layer < 4 else 3 * 64)
        g, w = got_w[lo:hi], want_w[lo:hi]
        err = np.linalg.norm(g - w) / (np.linalg.norm(w) + 1e-30)
        assert err < 3e-2, (layer, err)
    assert np.all(got_w[4 * 4096 + 3 * 64:] == 0.0)
    touched = want_t != 0.0
    err = np.linalg.norm(got_t[touched] - want_t[touched]) / np.linalg.norm(want_t[touched])
    assert err < 5e-2, err
    assert np.count_nonzero(got_t[~touched]) == 0


@pytest.mark.gpu
def test_adam_bit_exact(trained):
    import torch
    q = make_queries(3000, seed=4)
    t = target_function(q)
    trained.gradients(torch.from_numpy(q).cuda(), torch.from_numpy(t).cuda())
    torch.cuda.synchronize()
    before = {k: host_region(trained, k, torch.float32).copy()
              for k in ("weights", "weight_m", "weight_v", "weight_grad", "table", "table_m", "table_v", "table_grad")}
    s0 = trained.scalars()
    trained.adam()
    torch.cuda.synchronize()
    s1 = trained.scalars()
    assert s1.step == s0.step + 1
    b1 = np.float32(np.float32(s0.beta1_power) * np.float32(trained.cfg.beta1))
    b2 = np.float32(np.float32(s0.beta2_power) * np.float32(trained.cfg.beta2))
    assert np.float32(s1.beta1_power) == b1 and np.float32(s1.beta2_power) == b2
    lib = ob.load()
    for w, m, v, g, count in (("weights", "weight_m", "weight_v", "weight_grad", abi.CACHE_WEIGHTS),
                              ("table", "table_m", "table_v", "table_grad", before["table"].size)):
        ww, mm, vv = before[w][:count].copy(), before[m][:count].copy(), before[v][:count].copy()
        gg = before[g][:count].copy()
        lib.oracle_cache_adam(C.byref(trained.cfg), count, ww.ctypes.data, mm.ctypes.data, vv.ctypes.data,
                              gg.ctypes.data, C.c_float(b1), C.c_float(b2))
        got = host_region(trained, w, torch.float32)[:count]
        if w == "weights":
            live = np.ones(count, bool)
            live[4 * 4096 + 3 * 64:] = False  # the output layer's padding rows are not updated
            np.testing.assert_array_equal(got[live].view(np.uint32), ww[live].view(np.uint32))
            np.testing.assert_array_equal(got[~live], before[w][:count][~live])
        else:
            np.testing.assert_array_equal(got.view(np.uint32), ww.view(np.uint32))


@pytest.mark.gpu
def test_training_fits_target():
    import torch
    cache = small_cache(table_log2=14)
    q = make_queries(16384, seed=5)
    t = target_function(q)
    dq, dt = torch.from_numpy(q).cuda(), torch.from_numpy(t).cuda()
    losses = []
    for step in range(300):
        cache.train(dq, dt)
        if step in (0, 299):
            torch.cuda.synchronize()
            losses.append(cache.scalars().loss)
    s = cache.scalars()
    assert s.step == 300 and s.skipped_steps == 0
    assert losses[1] < 0.1 * losses[0], losses
    # Held-out points of the same function.
    hq = make_queries(4096, seed=6)
    pred = cache.forward(torch.from_numpy(hq).cuda()).cpu().numpy()[:, :3]
    ht = target_function(hq)[:, :3]
    rel = np.mean((pred - ht) ** 2 / (ht ** 2 + 0.01))
    # The untrained network starts near 20; 300 steps on 16,384 points
    # generalise to about 0.04.
    assert rel < 0.1, rel
    assert rb.status_flags() & 8 == 0


@pytest.mark.gpu
@pytest.mark.parametrize("cache_only", [0, 1])
def test_renderer_cache_forms_train_on_a_side_stream(cache_only):
    """The renderer's radiance-cache forms (GI passes with the cache, and the
    cache-only GI): training runs on a side stream overlapping the frame and
    joins before it ends; the frames stay finite, the cache trains (step count
    advances) and its pass is timed."""
    import torch
    from tests.helpers import make_scene
    setup = make_scene(rb.SCENE_COURTYARD, 0, 20000)
    settings = setup.settings
    settings.radiance_cache = 1
    settings.cache_only_gi = cache_only
    settings.cache_training_samples = 4096
    renderer = rb.Renderer(settings)
    renderer.set_scene(setup.mesh)
    frame = rb.frame_input(setup.mesh, 160, 96)
    for _ in range(6):
        renderer.render(frame)
    renderer.synchronize()
    assert rb.status_flags() & 8 == 0
    params, plan, _ = renderer.last_frame()
    assert plan.gi_from_cache == cache_only and params.radiance_cache == 1.0
    hdr = renderer.download("display.hdr", np.float16)[:160 * 96 * 4].astype(np.float32)
    assert np.all(np.isfinite(hdr))
    gi = renderer.download("gi.color0", np.float16).astype(np.float32)
    assert np.count_nonzero(gi) > 0
    times = renderer.pass_history(3)
    cache_index = rb.PASS_NAMES.index("cache")
    assert np.all(times[:, cache_index] > 0.0)
    layout = rb.cache_layout(rb.cache_config())
    pointer, nbytes = renderer.buffer("cache.state")
    raw = rb.device_view(pointer, nbytes, torch.uint8)[layout.scalars:layout.scalars + 64].cpu().numpy()
    scalars = rb.abi.RestirCacheScalars.from_buffer_copy(raw[:C.sizeof(rb.abi.RestirCacheScalars)].tobytes())
    assert scalars.step == 6
    if not cache_only:
        # The GI passes with the cache store no reservoir weight above 64.
        gi_pixels = params.gi_width * params.gi_height
        for name in ("gi.receiver0", "gi.receiver1"):
            weights = renderer.download(name, np.float32)[:4 * gi_pixels].reshape(-1, 4)[:, 3]
            assert np.all(np.isfinite(weights)) and weights.max() <= 64.0, name


@pytest.mark.gpu
def test_training_is_reproducible_bit_for_bit():
    """Two caches from the same seed, trained on the same batches, stay equal
    bit for bit: the weight gradients are summed in block order and the hash
    table's gradient in 64-bit fixed point, so no step depends on the order in
    which the samples' scattered contributions arrive (a 4,096-entry table
    and 65,536 samples give every entry many colliding contributions)."""
    import torch
    caches = [small_cache(), small_cache()]
    q = make_queries(65536, seed=11)
    t = target_function(q)
    dq, dt = torch.from_numpy(q).cuda(), torch.from_numpy(t).cuda()
    for step in range(25):
        for cache in caches:
            cache.train(dq, dt)
        if step in (0, 24):
            torch.cuda.synchronize()
            for name in ("table_grad", "weight_grad", "table", "weights"):
                a = host_region(caches[0], name, torch.int32)
                b = host_region(caches[1], name, torch.int32)
                assert np.array_equal(a, b), (step, name)
    assert caches[0].scalars().skipped_steps == 0
    assert np.count_nonzero(host_region(caches[0], "table_grad", torch.float32)) > 1000
