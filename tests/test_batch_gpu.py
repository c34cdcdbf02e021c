"""Batches of views (restir_batch_*): every view of a batch frame equals what
a renderer of that view alone produces, bit for bit, although the views share
one shadow atlas and one GI ray queue traced by one persistent launch; the
queue tracer gives the same hits at every launch shape the autotuner tries."""
import ctypes as C

import numpy as np
import pytest

import oracle.binding as ob
import restir_b200 as rb
from tests.helpers import make_scene, seeded_rays

SIZES = [(160, 90), (96, 96), (200, 120)]


def batch_setup():
    mesh = rb.Mesh.procedural(rb.SCENE_COURTYARD, 0, 20000)
    settings = rb.default_settings(mesh)
    settings.grid_mode = rb.GRID_DETERMINISTIC
    settings.extra_lights = 16
    base = rb.frame_input(mesh, 64, 64)
    inputs = []
    for v, (w, h) in enumerate(SIZES):
        inputs.append(rb.frame_input(mesh, w, h, yaw=base.yaw + 0.35 * v, pitch=base.pitch - 0.05 * v))
    return mesh, settings, inputs


@pytest.mark.gpu
def test_batch_views_equal_single_renderers():
    mesh, settings, inputs = batch_setup()
    batch = rb.Batch(settings, len(inputs))
    batch.set_scene(mesh)
    frames = 3
    for _ in range(frames):
        batch.render(inputs)
    batch.synchronize()
    rb.status_flags()
    for v, frame in enumerate(inputs):
        single = rb.Renderer(settings)
        single.set_scene(mesh)
        for _ in range(frames):
            single.render(frame)
        single.synchronize()
        for name, dtype in (("hdr", np.uint16), ("gi.sample0", np.float32), ("gi.sample1", np.float32),
                            ("di.diffuse", np.uint16), ("gbuffer.depth", np.float32)):
            got = batch.download(v, name, dtype)
            want = single.download(name, dtype)
            assert got.shape == want.shape, name
            np.testing.assert_array_equal(got.view(np.uint8), want.view(np.uint8), err_msg=f"view {v} {name}")
        hdr = single.download("hdr", np.uint16).reshape(-1, 4)
        assert np.count_nonzero(hdr[:, :3]) > 0.2 * hdr[:, :3].size
        single.close()
    params, _, _ = batch.last_frame(2)
    assert (params.width, params.height) == SIZES[2]
    assert rb.status_flags() & (1 | 4) == 0
    batch.close()


@pytest.mark.gpu
def test_batch_autotune_picks_a_shape():
    mesh, settings, inputs = batch_setup()
    batch = rb.Batch(settings, len(inputs))
    batch.set_scene(mesh)
    best = batch.autotune(inputs, frames=2)
    assert best.tracer_threads in (64, 128, 256) and best.ms_per_frame > 0.0
    t = batch.tuning
    assert (t.tracer_threads, t.tracer_blocks_per_sm) == (best.tracer_threads, best.tracer_blocks_per_sm)
    bad = rb.abi.RestirBatchTuning(96, 0, 0.0)
    assert rb.load().restir_batch_set_tuning(batch.handle, C.byref(bad)) == rb.ERROR_INVALID_ARGUMENT
    batch.close()


@pytest.mark.gpu
@pytest.mark.parametrize("threads,blocks", [(64, 0), (128, 0), (256, 0), (128, 2), (256, 1)])
def test_trace_queue_shapes_bit_exact(threads, blocks):
    """restir_trace_queue over a filled queue: the oracle's closest hits at every shape."""
    import torch
    setup = make_scene(rb.SCENE_COURTYARD, 0, 100000)
    rays = seeded_rays(setup, 50000, seed=21)
    n = len(rays)
    lib = rb.load()
    nbytes = int(lib.restir_ray_queue_bytes(n))
    queue = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
    up = lambda b: (b + 255) // 256 * 256
    queue[256:256 + 32 * n] = torch.from_numpy(rays.view(np.uint8).reshape(-1)).cuda()
    queue[0:4] = torch.from_numpy(np.array([n], np.uint32).view(np.uint8)).cuda()
    rb.check(lib.restir_trace_queue(setup.device_scene(), queue.data_ptr(), n, threads, blocks, None), "trace_queue")
    torch.cuda.synchronize()
    tri_at = 256 + up(32 * n)
    dist_at = tri_at + up(4 * n)
    got_ids = queue[tri_at:tri_at + 4 * n].cpu().numpy().view(np.int32)
    got_t = queue[dist_at:dist_at + 4 * n].cpu().numpy().view(np.float32)
    ids = np.zeros(n, np.int32)
    t = np.zeros(n, np.float32)
    ob.load().oracle_trace(None, setup.host_scene(), rays.ctypes.data, ids.ctypes.data, t.ctypes.data, n,
                           rb.TRACE_CLOSEST)
    np.testing.assert_array_equal(got_ids, ids)
    np.testing.assert_array_equal(got_t.view(np.uint32), t.view(np.uint32))
    assert lib.restir_trace_queue(setup.device_scene(), queue.data_ptr(), n, 96, 0, None) == rb.ERROR_INVALID_ARGUMENT
