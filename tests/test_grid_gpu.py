"""The hash grid passes on the GPU against the oracle (cs_grid_clear.sc,
cs_grid_insert.sc): in the deterministic mode every cell's count and entry
list are bit-exact; in the atomic mode counts are exact and entry lists equal
as multisets."""
import numpy as np
import pytest

import oracle.binding as ob
import restir_b200 as rb
from tests.helpers import gbuffer_struct, grid_cells, host_gbuffer, make_scene, params_for, to_device


def run_grid(setup, params, gbuffer_host):
    import torch
    T, Cap = params.grid_table_size, params.grid_cell_capacity
    host = np.zeros(T * (2 + Cap), np.uint32)
    ob.load().oracle_grid_clear(params, host.ctypes.data)
    ob.load().oracle_grid_insert(params, gbuffer_struct(gbuffer_host), host.ctypes.data)
    dev = torch.full((T * (2 + Cap),), 7, dtype=torch.int32, device="cuda")
    gb_dev = to_device(gbuffer_host)
    rb.check(rb.load().restir_grid_clear(params, dev.data_ptr(), None), "grid clear")
    rb.check(rb.load().restir_grid_insert(params, gbuffer_struct(gb_dev), dev.data_ptr(), None), "grid insert")
    torch.cuda.synchronize()
    return host, dev.cpu().numpy().view(np.uint32)


@pytest.mark.gpu
@pytest.mark.parametrize("scene,size,table", [((rb.SCENE_CORNELL, 0), (256, 256), 1 << 16),
                                              ((rb.SCENE_COURTYARD, 100000), (640, 360), 1 << 20),
                                              ((rb.SCENE_CITY, 200000), (640, 360), 1 << 15)])
@pytest.mark.parametrize("mode", [rb.GRID_DETERMINISTIC, rb.GRID_ATOMIC])
def test_grid_insert(scene, size, table, mode):
    setup = make_scene(*scene)
    w, h = size
    params, _ = params_for(setup, w, h, grid_table_size=table, grid_mode=mode, gi_divisor=1 if w <= 256 else 2)
    gb = host_gbuffer(w, h)
    ob.load().oracle_gbuffer_primary(params, setup.host_scene(), gbuffer_struct(gb))
    host, dev = run_grid(setup, params, gb)
    T, Cap = params.grid_table_size, params.grid_cell_capacity
    hc = grid_cells(host, T, Cap)
    dc = grid_cells(dev, T, Cap)
    assert set(hc) == set(dc)
    assert len(hc) > 10
    for key, (count, entries) in hc.items():
        dcount, dentries = dc[key]
        assert dcount == count
        if mode == rb.GRID_DETERMINISTIC:
            np.testing.assert_array_equal(dentries, entries)
        elif count <= Cap:
            np.testing.assert_array_equal(np.sort(dentries), np.sort(entries))
    # No probe sequence ran out.
    assert rb.status_flags() & 2 == 0
