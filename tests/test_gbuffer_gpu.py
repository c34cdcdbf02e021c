"""The G-buffer primary rays and the shadow atlas on the GPU against the
oracle, bit for bit."""
import numpy as np
import pytest

import oracle.binding as ob
import restir_b200 as rb
from tests.helpers import gbuffer_struct, host_gbuffer, make_scene, params_for, to_device, to_host


def render_gbuffer(setup, params, w, h):
    host = host_gbuffer(w, h)
    ob.load().oracle_gbuffer_primary(params, setup.host_scene(), gbuffer_struct(host))
    dev = to_device(host_gbuffer(w, h))
    rb.check(rb.load().restir_gbuffer_primary(params, setup.device_scene(), gbuffer_struct(dev), None), "gbuffer")
    return host, to_host(dev)


@pytest.mark.gpu
@pytest.mark.parametrize("scene,size", [((rb.SCENE_CORNELL, 0), (256, 256)), ((rb.SCENE_COURTYARD, 100000), (320, 180)),
                                        ((rb.SCENE_CITY, 200000), (331, 187))])
def test_gbuffer_bit_exact(scene, size):
    setup = make_scene(*scene)
    w, h = size
    params, _ = params_for(setup, w, h)
    host, dev = render_gbuffer(setup, params, w, h)
    for name in host:
        np.testing.assert_array_equal(dev[name], host[name], err_msg=name)
    assert (host["depth"] < 1.0).mean() > 0.2


@pytest.mark.gpu
@pytest.mark.parametrize("scene", [(rb.SCENE_CORNELL, 0), (rb.SCENE_COURTYARD, 100000)])
def test_shadow_atlas_bit_exact(scene):
    import torch
    setup = make_scene(*scene)
    params, _ = params_for(setup, 64, 64, shadow_face_size=256)
    f = params.shadow_face_size
    host = np.zeros(6 * f * f, np.float32)
    ob.load().oracle_shadow_atlas(params, setup.host_scene(), host.ctypes.data)
    dev = torch.zeros(6 * f * f, dtype=torch.float32, device="cuda")
    rb.check(rb.load().restir_shadow_atlas(params, setup.device_scene(), dev.data_ptr(), None), "shadow")
    np.testing.assert_array_equal(dev.cpu().numpy().view(np.uint32), host.view(np.uint32))
    assert (host < 1.0).mean() > 0.5
