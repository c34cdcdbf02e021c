"""The allocation-free error pass, restir_error_noalloc.

Some callers of this library cannot allocate device memory when they run the
error pass: an engine whose own memory manager owns the whole device budget,
or a real-time loop that must not enter the driver's allocator (cudaMalloc and
cudaFree can synchronise the device). For them the library keeps the pass's scratch (the
per-block FP64 partial records) in a fixed 64 KB array of its own, and the
entry point takes only inputs and the output.

This file is named to run last, so that a run stopping at the first failure
has already run every other test. It checks, through the C ABI, that two
calls in a row give the same records as restir_error (caller scratch) within
the tolerance of the other FP64 error tests (the two differ only in how many
blocks share the sum, so in summation order), and that images beyond the
array's limit are refused.
"""
import ctypes as C

import numpy as np
import pytest

import restir_b200 as rb
from restir_b200.abi import RestirParams

TOO_LARGE = -7


def make_inputs(torch, width, height, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    n = width * height
    display = (torch.rand(n * 4, generator=g, device="cuda") * 4.0).to(torch.float16).view(torch.int16)
    mean = torch.rand(3 * n, generator=g, device="cuda", dtype=torch.float64) * 4.0
    alpha = (torch.rand(n, generator=g, device="cuda") < 0.8).to(torch.uint8)
    return display, mean, alpha


def params_of(width, height):
    p = RestirParams()
    p.width, p.height = width, height
    return p


@pytest.mark.gpu
def test_noalloc_error_matches_caller_scratch_on_two_calls():
    import torch
    lib = rb.load()
    lib.restir_error_noalloc.restype = C.c_int
    lib.restir_error_noalloc.argtypes = [C.POINTER(RestirParams), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p]
    for call, (width, height, seed) in enumerate(((1920, 1080, 1), (1280, 720, 2))):
        params = params_of(width, height)
        display, mean, alpha = make_inputs(torch, width, height, seed)
        scratch = torch.zeros(lib.restir_error_scratch_bytes(width, height) // 8 + 1, dtype=torch.float64,
                              device="cuda")
        want = torch.zeros(4, dtype=torch.float64, device="cuda")
        got = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
        rb.check(lib.restir_error(params, display.data_ptr(), mean.data_ptr(), alpha.data_ptr(), want.data_ptr(),
                                  scratch.data_ptr(), None), "restir_error")
        rb.check(lib.restir_error_noalloc(params, display.data_ptr(), mean.data_ptr(), alpha.data_ptr(),
                                          got.data_ptr(), None), f"restir_error_noalloc (call {call + 1})")
        torch.cuda.synchronize()
        want, got = want.cpu().numpy(), got.cpu().numpy()
        assert want[3] == got[3] == float(alpha.sum().item())
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=0)


@pytest.mark.gpu
def test_noalloc_error_refuses_images_beyond_its_scratch():
    import torch
    lib = rb.load()
    lib.restir_error_noalloc.restype = C.c_int
    lib.restir_error_noalloc.argtypes = [C.POINTER(RestirParams), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p]
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda")
    # 4096 x 4096 = 16.7M pixels, beyond the 8,388,608-pixel limit: refused before any launch.
    status = lib.restir_error_noalloc(params_of(4096, 4096), dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(),
                                      dummy.data_ptr(), None)
    assert status == TOO_LARGE
