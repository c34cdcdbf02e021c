"""The oracle against the committed known-answer fixtures (tests/golden,
made by tests/golden/make_golden.py), and the device hashes against them."""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle.binding as ob
import restir_b200 as rb

GOLDEN = Path(__file__).resolve().parent / "golden"


def _eval(fn, bits):
    x = np.asarray(bits, np.uint64).astype(np.uint32).view(np.float32)
    out = np.zeros_like(x)
    ob.load().oracle_numeric_eval(fn, x.ctypes.data, out.ctypes.data, len(x))
    return out.view(np.uint32)


def test_hash_kat():
    kat = json.loads((GOLDEN / "hash_kat.json").read_text())
    np.testing.assert_array_equal(_eval(8, kat["input"]), np.array(kat["pcg"], np.uint64).astype(np.uint32))
    np.testing.assert_array_equal(_eval(9, kat["input"]), np.array(kat["checksum"], np.uint64).astype(np.uint32))


def test_grid_key_kat():
    g = np.load(GOLDEN / "grid_keys.npz")
    n = len(g["positions"])
    cell, slot, checksum = (np.zeros(n, np.uint32) for _ in range(3))
    pos = np.ascontiguousarray(g["positions"])
    nrm = np.ascontiguousarray(g["normals"])
    rnd = np.ascontiguousarray(g["randoms"])
    cam = np.ascontiguousarray(g["camera"])
    const = np.ascontiguousarray(g["constants"])
    ob.load().oracle_grid_keys(cam.ctypes.data, const.ctypes.data, int(g["table_mask"]) + 1, pos.ctypes.data,
                               nrm.ctypes.data, rnd.ctypes.data, n, cell.ctypes.data, slot.ctypes.data,
                               checksum.ctypes.data)
    np.testing.assert_array_equal(cell, g["cell_bits"])
    np.testing.assert_array_equal(slot, g["slot"])
    np.testing.assert_array_equal(checksum, g["checksum"])


@pytest.mark.gpu
def test_device_hash_kat():
    import torch
    kat = json.loads((GOLDEN / "hash_kat.json").read_text())
    x = np.array(kat["input"], np.uint64).astype(np.uint32).view(np.float32)
    for fn, key in ((8, "pcg"), (9, "checksum")):
        d_in = torch.from_numpy(x.copy()).cuda()
        d_out = torch.empty_like(d_in)
        rb.check(rb.load().restir_numeric_eval(fn, d_in.data_ptr(), d_out.data_ptr(), len(x), None), "numeric")
        torch.cuda.synchronize()
        np.testing.assert_array_equal(d_out.cpu().numpy().view(np.uint32),
                                      np.array(kat[key], np.uint64).astype(np.uint32))
