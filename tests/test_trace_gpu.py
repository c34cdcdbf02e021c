"""BVH traversal on the GPU (restir_trace) against the oracle's restatement of
shaders/bvh.sh: hit triangle ids and distances bit-exact, on our builder's
buffer and on the buffer the reference's own builder produced."""
from pathlib import Path

import numpy as np
import pytest

import oracle.binding as ob
import restir_b200 as rb
from tests.helpers import make_scene, seeded_rays

GOLDEN = Path(__file__).resolve().parent / "golden"
KINDS = [rb.TRACE_CLOSEST, rb.TRACE_ANY, rb.TRACE_CLOSEST_STACKLESS, rb.TRACE_CLOSEST_WATERTIGHT,
         rb.TRACE_CLOSEST_QUEUE, rb.TRACE_ANY_WAVE]


def trace_both(setup, rays, kind, scene_host=None, scene_dev=None):
    import torch
    n = len(rays)
    host_scene = scene_host or setup.host_scene()
    ids = np.zeros(n, np.int32)
    t = np.zeros(n, np.float32)
    ob.load().oracle_trace(None, host_scene, rays.ctypes.data, ids.ctypes.data, t.ctypes.data, n, kind)
    d_rays = torch.from_numpy(rays).cuda()
    d_ids = torch.empty(n, dtype=torch.int32, device="cuda")
    d_t = torch.empty(n, dtype=torch.float32, device="cuda")
    rb.check(rb.load().restir_trace(None, scene_dev or setup.device_scene(), d_rays.data_ptr(), d_ids.data_ptr(),
                                    d_t.data_ptr(), n, kind, None), "restir_trace")
    torch.cuda.synchronize()
    return ids, t, d_ids.cpu().numpy(), d_t.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("scene", [(rb.SCENE_CORNELL, 0), (rb.SCENE_COURTYARD, 100000), (rb.SCENE_CITY, 200000)])
@pytest.mark.parametrize("kind", KINDS)
def test_trace_bit_exact(scene, kind):
    setup = make_scene(*scene)
    rays = seeded_rays(setup, 1 << 16, seed=11)
    ids, t, d_ids, d_t = trace_both(setup, rays, kind)
    np.testing.assert_array_equal(d_ids, ids)
    np.testing.assert_array_equal(d_t.view(np.uint32), t.view(np.uint32))
    assert (ids >= 0).mean() > 0.2
    assert rb.status_flags() == 0


@pytest.mark.gpu
def test_trace_on_reference_built_buffer():
    import torch
    g = np.load(GOLDEN / "reference_cornell.npz")
    setup = make_scene(rb.SCENE_CORNELL)
    nodes, offset, _ = (int(v) for v in g["header"])
    bvh = np.ascontiguousarray(g["bvh"])
    host = setup.host_scene()
    host.bvh, host.node_count, host.triangle_offset = bvh.ctypes.data, nodes, offset
    d_bvh = torch.from_numpy(bvh).cuda()
    dev = setup.device_scene()
    dev.bvh, dev.node_count, dev.triangle_offset = d_bvh.data_ptr(), nodes, offset
    rays = seeded_rays(setup, 1 << 16, seed=12)
    for kind in KINDS:
        ids, t, d_ids, d_t = trace_both(setup, rays, kind, host, dev)
        np.testing.assert_array_equal(d_ids, ids)
        np.testing.assert_array_equal(d_t.view(np.uint32), t.view(np.uint32))


@pytest.mark.gpu
def test_watertight_agrees_with_moeller_trumbore_off_edges():
    setup = make_scene(rb.SCENE_COURTYARD, 0, 100000)
    rays = seeded_rays(setup, 1 << 16, seed=13)
    ids_mt, t_mt, _, _ = trace_both(setup, rays, rb.TRACE_CLOSEST)
    ids_wt, t_wt, _, _ = trace_both(setup, rays, rb.TRACE_CLOSEST_WATERTIGHT)
    both = (ids_mt >= 0) & (ids_wt >= 0)
    # Where the two tests pick different triangles, the scene has coplanar
    # faces (box bottoms on the ground): the distances still agree.
    assert (ids_mt == ids_wt).mean() > 0.98
    assert ((ids_mt >= 0) == (ids_wt >= 0)).mean() > 0.9999
    # The two tests round differently: relative 1e-5 for distant hits, and an
    # absolute floor (a few float ulps of the scene's coordinates) for hits
    # next to the ray origin, where the difference o - v0 cancels.
    np.testing.assert_allclose(t_wt[both], t_mt[both], rtol=1e-5, atol=4e-6 * setup.mesh.desc.radius)


@pytest.mark.gpu
def test_empty_ray_set_and_invalid_arguments():
    setup = make_scene(rb.SCENE_CORNELL)
    lib = rb.load()
    assert lib.restir_trace(None, setup.device_scene(), 0, 0, 0, 0, rb.TRACE_CLOSEST, None) == -1
    import torch
    d = torch.zeros(8, device="cuda")
    i = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.restir_trace(None, setup.device_scene(), d.data_ptr(), i.data_ptr(), d.data_ptr(), 0,
                            rb.TRACE_CLOSEST, None) == 0
    assert lib.restir_trace(None, setup.device_scene(), d.data_ptr(), i.data_ptr(), d.data_ptr(), 1, 9, None) == -1


def test_oracle_wave_walk_matches_stackless_any_hit():
    """The oracle's lock-step walk (bvh.sh:177-212) gives each lane the
    stackless walk's any hit (bvh.sh:140-174): same triangles, same distances."""
    setup = make_scene(rb.SCENE_COURTYARD, 0, 20000)
    rays = seeded_rays(setup, 1 << 12, seed=14)
    host = setup.host_scene()
    out = {}
    for kind in (rb.TRACE_ANY, rb.TRACE_ANY_WAVE):
        ids = np.zeros(len(rays), np.int32)
        t = np.zeros(len(rays), np.float32)
        ob.load().oracle_trace(None, host, rays.ctypes.data, ids.ctypes.data, t.ctypes.data, len(rays), kind)
        out[kind] = (ids, t)
    np.testing.assert_array_equal(out[rb.TRACE_ANY_WAVE][0], out[rb.TRACE_ANY][0])
    np.testing.assert_array_equal(out[rb.TRACE_ANY_WAVE][1].view(np.uint32), out[rb.TRACE_ANY][1].view(np.uint32))
    assert (out[rb.TRACE_ANY][0] >= 0).mean() > 0.2
