"""The oracle's own scene set-up and frame uniforms (oracle/workload.py,
oracle/oracle_frame.cpp), which the CPU arm of the benchmark runs without the
product's library, against the product's: the same procedural scene, the
reference builder's BVH equal to the product builder's, the reference's
light list, and frame uniforms equal bit for bit over frames that carry
state (TAA jitter, history, reference mode)."""
import ctypes as C

import numpy as np
import pytest

import oracle.binding as ob
import restir_b200 as rb
from tests.helpers import make_scene

pytestmark = pytest.mark.skipif(not ob.reference_available(), reason="oracle/_ref/libref_bvh.so not built")


def test_settings_defaults_equal():
    from oracle.workload import OracleSetup
    setup = OracleSetup(rb.SCENE_CORNELL)
    want = rb.default_settings(rb.Mesh.procedural(rb.SCENE_CORNELL))
    assert bytes(setup.settings) == bytes(want)


@pytest.mark.parametrize("scene", [(rb.SCENE_CORNELL, 0, 0), (rb.SCENE_COURTYARD, 2, 30000), (rb.SCENE_CITY, 3, 60000)])
def test_scene_bvh_and_lights_equal_the_products(scene):
    from oracle.workload import OracleSetup
    oracle_setup = OracleSetup(*scene, extra_lights=64)
    product = make_scene(*scene, extra_lights=64)
    assert oracle_setup.mesh.triangle_count == product.mesh.triangle_count
    n = product.mesh.triangle_count
    np.testing.assert_array_equal(oracle_setup.mesh.array("positions", C.c_float, 9 * n), product.mesh.positions())
    np.testing.assert_array_equal(oracle_setup.materials, product.materials)
    # The reference's builder and the product's give the same buffer, slot order and normals.
    np.testing.assert_array_equal(oracle_setup.bvh.data.view(np.uint32), product.bvh.data.view(np.uint32))
    np.testing.assert_array_equal(oracle_setup.bvh.order, product.bvh.order)
    np.testing.assert_array_equal(oracle_setup.bvh.triangle_normals, product.bvh.triangle_normals)
    assert oracle_setup.lights.count == product.lights.count
    np.testing.assert_array_equal(oracle_setup.lights.data[:16 * product.lights.count],
                                  product.lights.data[:16 * product.lights.count])


def test_frame_uniforms_equal_the_products():
    """oracle_frame_params / oracle_frame_advance against restir_frame_params /
    restir_frame_advance: 1080p and 720p views, TAA jitter over its 8-frame
    cycle, half- and full-resolution GI, the reference mode's overrides and
    1024-frame jitter, a moving camera."""
    from oracle.frame import ProductHost
    from oracle.workload import OracleHost, OracleSetup
    setup = OracleSetup(rb.SCENE_CITY, 0, 60000, extra_lights=64)
    oracle_host, product_host = OracleHost(), ProductHost()
    product_mesh = rb.Mesh.procedural(rb.SCENE_CITY, 0, 60000)
    for (w, h), divisor in (((1920, 1080), 2), ((1280, 720), 1)):
        settings = setup.settings
        settings.gi_divisor = divisor
        states = [rb.initial_state(), rb.initial_state()]
        for frame in range(12):
            fi = rb.frame_input(product_mesh, w, h, yaw=product_mesh.desc.camera_yaw + 0.01 * (frame // 4))
            if frame == 6:
                for s in states:
                    s.reference_accumulating = 1
            got = oracle_host.frame_params(settings, setup.mesh, setup.lights.count, setup.bvh, fi, states[0])
            want = product_host.frame_params(settings, product_mesh, setup.lights.count, setup.bvh, fi, states[1])
            assert bytes(got[0]) == bytes(want[0]), (w, frame)
            assert bytes(got[1]) == bytes(want[1]), (w, frame)
            oracle_host.advance(*got, fi, states[0])
            product_host.advance(*want, fi, states[1])
            assert bytes(states[0]) == bytes(states[1])
            d = [host.display_params(C.cast((C.c_float * 16)(*got[0].inv_view_proj), C.c_void_p),
                                     C.cast((C.c_float * 16)(*states[0].previous_unjittered_view_proj), C.c_void_p),
                                     w, h, got[1].taa, states[0].taa_valid, 1, frame % 2, 1.5, 1.0 / 60.0, 0.5, 1, 0, 0)
                 for host in (oracle_host, product_host)]
            assert bytes(d[0]) == bytes(d[1])


def test_oracle_only_frames_equal_product_set_up_frames():
    """Two frames through the oracle's passes, one run set up by the product's
    host code and one by the oracle's alone: every target equal."""
    from oracle.frame import FrameRunner
    from oracle.workload import OracleSetup
    oracle_setup = OracleSetup(rb.SCENE_COURTYARD, 1, 20000, extra_lights=16)
    product = make_scene(rb.SCENE_COURTYARD, 1, 20000, extra_lights=16)
    runs = []
    for setup in (oracle_setup, product):
        setup.settings.grid_mode = rb.GRID_DETERMINISTIC
        runner = FrameRunner(setup, 96, 64, "oracle", setup.settings)
        for _ in range(2):
            runner.render()
        runs.append(runner)
    for name in runs[0].buffers:
        np.testing.assert_array_equal(runs[0].host(name), runs[1].host(name), err_msg=name)
    assert np.count_nonzero(runs[0].host("display")) > 0


def test_lit_city_has_4096_emissive_triangles():
    """RESTIR_SCENE_CITY_LIT, the stress configuration's scene: the city with
    2,048 emissive panels, so the light list holds 4,096 emissive triangles
    (plus the extra point lights); the oracle's copy of the generator agrees."""
    from oracle.workload import OracleSetup
    setup = OracleSetup(rb.SCENE_CITY_LIT, 0, 200_000, extra_lights=1024)
    assert setup.lights.triangles == 4096 and setup.lights.count == 4096 + 1024
    product = make_scene(rb.SCENE_CITY_LIT, 0, 200_000, extra_lights=1024)
    assert product.lights.count == setup.lights.count
    np.testing.assert_array_equal(setup.lights.data, product.lights.data)
