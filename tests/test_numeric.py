"""The ABI's numeric conventions (include/restir_numeric.h): accuracy of the
host implementation against numpy, and bit-identity of the device's."""
import numpy as np
import pytest

import oracle.binding as ob
import restir_b200 as rb


def host_eval(fn, x):
    out = np.zeros_like(x)
    ob.load().oracle_numeric_eval(fn, x.ctypes.data, out.ctypes.data, len(x))
    return out


def test_sincos_accuracy():
    x = np.linspace(-7.0, 14.0, 200001, dtype=np.float32)
    s, c = host_eval(0, x), host_eval(1, x)
    assert np.max(np.abs(s.astype(np.float64) - np.sin(x.astype(np.float64)))) < 4e-7
    assert np.max(np.abs(c.astype(np.float64) - np.cos(x.astype(np.float64)))) < 4e-7


def test_exp_accuracy():
    x = np.linspace(-100.0, 80.0, 200001, dtype=np.float32)
    y = host_eval(2, x).astype(np.float64)
    ref = np.exp(x.astype(np.float64))
    normal = ref > 1.2e-38
    assert np.max(np.abs(y[normal] / ref[normal] - 1.0)) < 4e-7
    assert host_eval(2, np.array([-200.0, 200.0, np.nan], np.float32))[0] == 0.0
    assert np.isinf(host_eval(2, np.array([200.0], np.float32))[0])


def test_half_round_trip_matches_numpy():
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.normal(size=100000).astype(np.float32) * 10.0,
                        rng.normal(size=10000).astype(np.float32) * 1e-5,
                        np.array([0.0, -0.0, 65504.0, 65520.0, 1e-8, 6e-8, 3e-8, 2.98e-8], np.float32)])
    ref = x.astype(np.float16).astype(np.float32)
    np.testing.assert_array_equal(host_eval(4, x).view(np.uint32), ref.view(np.uint32))


def test_half_to_float_exhaustive():
    # Every binary16 pattern (denormals, infinities and NaN payloads included)
    # against numpy's widening, bit for bit.
    bits = np.arange(65536, dtype=np.uint32)
    out = host_eval(10, bits.view(np.float32).copy())
    expected = bits.astype(np.uint16).view(np.float16).astype(np.float32)
    np.testing.assert_array_equal(out.view(np.uint32), expected.view(np.uint32))


def test_log2_exp2_pow_accuracy():
    # The display passes' transcendental functions (auto exposure's log2,
    # tone mapping's exp2 and pow): a few ulps against float64.
    x = np.concatenate([np.geomspace(1e-44, 3e38, 200001).astype(np.float32),
                        np.linspace(0.5, 2.0, 50001, dtype=np.float32)])
    y = host_eval(11, x).astype(np.float64)
    ref = np.log2(x.astype(np.float64))
    assert np.max(np.abs(y - ref) / np.spacing(np.abs(ref).astype(np.float32))) < 4.0
    special = host_eval(11, np.array([0.0, -1.0, np.inf, np.nan, 1.0, 0.5], np.float32))
    assert special[0] == -np.inf and np.isnan(special[1]) and special[2] == np.inf and np.isnan(special[3])
    assert special[4] == 0.0 and special[5] == -1.0
    x = np.linspace(-160.0, 130.0, 400001, dtype=np.float32)
    y = host_eval(12, x).astype(np.float64)
    ref = np.exp2(x.astype(np.float64))
    normal = (ref > 1.2e-38) & (ref < 3.0e38)
    assert np.max(np.abs(y[normal] / ref[normal] - 1.0)) < 2e-7
    assert np.all(host_eval(12, np.array([-200.0, 0.0, 1.0, 128.0], np.float32)) == np.array([0.0, 1.0, 2.0, np.inf], np.float32))
    x = np.linspace(0.0, 4.0, 100001, dtype=np.float32)
    for fn, e in ((13, 2.2), (14, 1.0 / 2.2)):
        y = host_eval(fn, x).astype(np.float64)
        ref = x.astype(np.float64) ** e
        assert y[0] == 0.0
        assert np.max(np.abs(y[1:] / ref[1:] - 1.0)) < 4e-6


def test_unorm8_and_log2():
    x = np.linspace(-0.1, 1.1, 1201, dtype=np.float32)
    expected = np.round(np.clip(x, 0, 1).astype(np.float64) * 255.0 + 1e-9)
    np.testing.assert_array_equal(host_eval(5, x), np.floor(np.clip(x, 0, 1) * np.float32(255.0) + np.float32(0.5)))
    assert np.max(np.abs(host_eval(5, x) - expected)) <= 1.0
    v = np.array([1.0, 1.5, 2.0, 3.99, 4.0, 1024.0, 1e20], np.float32)
    np.testing.assert_array_equal(host_eval(6, v), np.floor(np.log2(v.astype(np.float64))))


@pytest.mark.gpu
def test_device_numeric_bit_identical():
    import torch
    rng = np.random.default_rng(2)
    inputs = {
        0: np.linspace(-7.0, 14.0, 100003, dtype=np.float32),
        1: np.linspace(-7.0, 14.0, 100003, dtype=np.float32),
        2: np.linspace(-110.0, 90.0, 100003, dtype=np.float32),
        3: rng.normal(size=100003).astype(np.float32) * 100.0,
        4: rng.normal(size=100003).astype(np.float32) * 100.0,
        5: np.linspace(-0.1, 1.1, 100003, dtype=np.float32),
        6: np.abs(rng.normal(size=100003).astype(np.float32)) * 1000.0 + 1.0,
        7: rng.random(100003).astype(np.float32),
        10: np.arange(65536, dtype=np.uint32).view(np.float32),
        11: np.geomspace(1e-44, 3e38, 100003).astype(np.float32),
        12: np.linspace(-160.0, 130.0, 100003, dtype=np.float32),
        13: np.linspace(0.0, 4.0, 100003, dtype=np.float32),
        14: np.linspace(0.0, 4.0, 100003, dtype=np.float32),
    }
    lib = rb.load()
    for fn, x in inputs.items():
        d_in = torch.from_numpy(x).cuda()
        d_out = torch.empty_like(d_in)
        rb.check(lib.restir_numeric_eval(fn, d_in.data_ptr(), d_out.data_ptr(), len(x), None), "numeric")
        torch.cuda.synchronize()
        host = host_eval(4 if fn == 3 else fn, x)
        np.testing.assert_array_equal(d_out.cpu().numpy().view(np.uint32), host.view(np.uint32), err_msg=f"fn {fn}")
