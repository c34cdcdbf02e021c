"""Failure detection: each guard of the device code trips on an input built
to trip it, the call returns with the status bit raised (restir_status), and
the next call is clean. Every input keeps every access in bounds and every
wait bounded, so no case can fault or hang the GPU:

  * bit 0, the traversal step cap (bvh.sh:23, kBvhMaxSteps = 2048): a BVH of
    two interior nodes whose links form a cycle of valid node indices (the
    root is its own right child and skip target; the second node's box is
    never hit and its skip link leads back to the root);
  * bit 1, the hash grid's probe cap (hashgrid.sh:56, 8 probes): a 16-slot
    table for a frame's thousands of cells;
  * bit 2, a full ray queue: a queue of 100 rays for a frame's candidates
    (rays past the capacity are dropped, not traced);
  * bit 3, the tensor-core steps' bounded wait: restir_cache_wait_check
    waits on an mbarrier no one arrives at, with no MMA issued.
"""
import ctypes as C

import numpy as np
import pytest

import oracle.binding as ob
import restir_b200 as rb
from restir_b200.abi import RestirGiHistory, RestirGiReservoirs, RestirScene
from tests.helpers import make_scene


def cyclic_bvh() -> np.ndarray:
    """Two nodes and one triangle (8 float4 rows). Node 0: a box around the
    rays, interior, right child 0, skip 0. Node 1: interior, a box far away,
    right child 0, skip 0. The stackless walk goes 0 -> 1 (box missed, skip)
    -> 0 -> ...; the short stack goes 0 -> right child 0 -> ...; both only
    ever read rows 0-3."""
    rows = np.zeros((8, 4), np.float32)
    rows[0] = (-10.0, -10.0, -10.0, 0.0)   # min, a = 0 (right child)
    rows[1] = (10.0, 10.0, 10.0, -1.0)     # max, b = -1 (interior, skip = -b - 1 = 0)
    rows[2] = (100.0, 100.0, 100.0, 0.0)
    rows[3] = (101.0, 101.0, 101.0, -1.0)
    rows[4] = (0.0, 0.0, 5.0, 0.0)         # the triangle (never reached)
    rows[5] = (1.0, 0.0, 5.0, 0.0)
    rows[6] = (0.0, 1.0, 5.0, 0.0)
    rows[7] = (0.5, 0.5, 0.5, 0.0)
    return rows.reshape(-1)


def scene_of(bvh, device: bool):
    import torch
    s = RestirScene()
    keep = torch.from_numpy(bvh).cuda() if device else bvh
    s.bvh = keep.data_ptr() if device else bvh.ctypes.data
    s.node_count, s.triangle_offset, s.triangle_count = 2, 4, 1
    return s, keep


def rays_inside(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = rng.uniform(-1.0, 1.0, (n, 3))
    rays[:, 3] = 5.0
    d = rng.normal(size=(n, 3))
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    return rays


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [rb.TRACE_CLOSEST, rb.TRACE_ANY, rb.TRACE_CLOSEST_STACKLESS,
                                  rb.TRACE_CLOSEST_QUEUE, rb.TRACE_ANY_WAVE])
def test_step_cap_stops_a_skip_link_cycle(kind):
    import torch
    lib = rb.load()
    rb.status_flags()  # clear
    bvh = cyclic_bvh()
    scene, keep = scene_of(bvh, device=True)
    rays = rays_inside(256, seed=kind)
    d_rays = torch.from_numpy(rays).cuda()
    ids = torch.full((len(rays),), 7, dtype=torch.int32, device="cuda")
    t = torch.zeros(len(rays), dtype=torch.float32, device="cuda")
    rb.check(lib.restir_trace(None, scene, d_rays.data_ptr(), ids.data_ptr(), t.data_ptr(), len(rays), kind, None),
             "restir_trace")
    torch.cuda.synchronize()
    assert rb.status_flags() & 1, "the step cap did not report the cycle"
    # No triangle was ever reached, the distance is the ray's tmax.
    assert (ids.cpu().numpy() == -1).all()
    np.testing.assert_array_equal(t.cpu().numpy(), rays[:, 3])
    # The oracle walks the same cycle to the same cap and result.
    want_ids = np.zeros(len(rays), np.int32)
    want_t = np.zeros(len(rays), np.float32)
    host_scene, _ = scene_of(bvh, device=False)
    ob.load().oracle_trace(None, host_scene, rays.ctypes.data, want_ids.ctypes.data, want_t.ctypes.data, len(rays),
                           kind)
    np.testing.assert_array_equal(ids.cpu().numpy(), want_ids)
    # The next call, on a sound BVH, is clean.
    setup = make_scene(rb.SCENE_CORNELL)
    rb.check(lib.restir_trace(None, setup.device_scene(), d_rays.data_ptr(), ids.data_ptr(), t.data_ptr(), len(rays),
                              kind, None), "restir_trace")
    torch.cuda.synchronize()
    assert rb.status_flags() == 0


@pytest.mark.gpu
def test_probe_cap_reports_a_full_grid():
    import torch
    from oracle.frame import FrameRunner
    lib = rb.load()
    setup = make_scene(rb.SCENE_COURTYARD, 0, 20000)
    runner = FrameRunner(setup, 96, 96, "cuda", setup.settings)
    runner.render()
    P = runner.params
    rb.status_flags()
    for table, expect in ((16, 2), (65536, 0)):
        P.grid_table_size = table
        grid = torch.zeros(table * (2 + P.grid_cell_capacity), dtype=torch.int32, device="cuda")
        rb.check(lib.restir_grid_clear(P, grid.data_ptr(), None), "grid clear")
        rb.check(lib.restir_grid_insert(P, runner.gbuffer(), grid.data_ptr(), None), "grid insert")
        torch.cuda.synchronize()
        assert rb.status_flags() & 2 == expect, table
        g = grid.cpu().numpy().view(np.uint32)
        # The small table is full: every slot holds a cell, no count overflowed the capacity's range.
        if table == 16:
            assert np.count_nonzero(g[:table]) == table


@pytest.mark.gpu
def test_full_ray_queue_drops_rays_and_reports():
    """The GI temporal wavefront with a queue of 100 rays for 2,304 BVH
    candidates: the rays past the capacity are dropped (their candidates count
    as misses), bit 2 is raised, and a queue of the full size is clean."""
    import torch
    from oracle.frame import FrameRunner
    lib = rb.load()
    setup = make_scene(rb.SCENE_CORNELL)
    settings = setup.settings
    settings.gi_divisor = 1
    settings.ray_mode = rb.RAY_BVH
    runner = FrameRunner(setup, 48, 48, "cuda", settings)
    runner.render()
    P, _ = runner.prepare()
    hr, hw = runner.history_read, 1 - runner.history_read
    history = RestirGiHistory(runner.b(f"gi.sample{hr}"), runner.b(f"gi.receiver{hr}"), runner.b(f"gi.normal{hr}"),
                              runner.b(f"gi.color{hr}"), runner.b(f"gi.moments{hr}"))
    out = RestirGiReservoirs(runner.b(f"gi.sample{hw}"), runner.b(f"gi.receiver{hw}"), runner.b(f"gi.normal{hw}"))
    records_bytes = int(lib.restir_gi_candidate_records_bytes(P))
    records = torch.zeros(records_bytes, dtype=torch.uint8, device="cuda")
    candidates = P.gi_width * P.gi_height * P.initial_candidates
    rb.status_flags()
    for capacity, expect in ((100, 4), (candidates, 0)):
        queue = torch.zeros(int(lib.restir_ray_queue_bytes(capacity)), dtype=torch.uint8, device="cuda")
        rb.check(lib.restir_ray_queue_reset(queue.data_ptr(), None), "queue reset")
        args = (P, runner.scene, runner.gbuffer(), history, runner.b(f"grid{hr}"), runner.b("atlas"),
                runner.b("gb.emissive"))
        rb.check(lib.restir_gi_temporal_candidates(*args, records.data_ptr(), records_bytes, queue.data_ptr(),
                                                   capacity, None), "candidates")
        rb.check(lib.restir_trace_queue(runner.scene, queue.data_ptr(), capacity, 128, 0, None), "trace queue")
        rb.check(lib.restir_gi_temporal_shade(*args, out, records.data_ptr(), records_bytes, queue.data_ptr(),
                                              capacity, None), "shade")
        torch.cuda.synchronize()
        assert rb.status_flags() & 4 == expect, capacity
        assert np.isfinite(runner.host(f"gi.receiver{hw}")).all()


@pytest.mark.gpu
def test_tensor_core_wait_gives_up_and_returns():
    import torch
    lib = rb.load()
    rb.status_flags()
    result = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    rb.check(lib.restir_cache_wait_check(64, result.data_ptr(), None), "restir_cache_wait_check")
    torch.cuda.synchronize()
    assert int(result.item()) == 0, "the wait did not give up"
    assert rb.status_flags() & 8
    # The context is usable and the cache's own tensor-core steps are clean afterwards.
    cache = rb.RadianceCache(rb.cache_config(bounds_min=(-1.0, -1.0, -1.0), bounds_max=(1.0, 1.0, 1.0)))
    q = torch.zeros((256, 16), dtype=torch.float32, device="cuda")
    q[:, 7] = 1.0
    q[:, 4:7] = torch.tensor([0.0, 1.0, 0.0], device="cuda")
    out = cache.query(q)
    torch.cuda.synchronize()
    assert torch.isfinite(out.float()).all()
    assert rb.status_flags() == 0
    assert lib.restir_cache_wait_check(0, result.data_ptr(), None) == rb.ERROR_INVALID_ARGUMENT
