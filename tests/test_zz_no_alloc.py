"""ispm_sblas_dot_noalloc: the dot product for callers that cannot let the
library allocate device memory (a fixed, pre-reserved budget; loops that must
not risk cudaMalloc's implicit synchronisation).  Its scratch is a static
device array in the library instead of a cudaMalloc'd area.

Called through the C ABI and compared with ispm_sblas_dot, the allocating
entry point, within the dot tests' tolerance (1e-13 of sum |x_i y_i| in FP64;
FP32 results equal up to the final FP32 rounding), on two calls in a row
(the second call runs on the scratch contents the first one left).

This file is collected last on purpose, so a stop-at-first-failure run has
executed every other test before it; it also passes on its own in a fresh
process."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _entry(ispm):
    L = ispm.lib_handle()
    f = L.ispm_sblas_dot_noalloc
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_int, ctypes.c_void_p]
    f.restype = ctypes.c_int
    g = L.ispm_sblas_dot
    g.argtypes = f.argtypes
    g.restype = ctypes.c_int
    return f, g


@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("n", [1, 1000, (1 << 21) + 3])
def test_noalloc_dot_matches_allocating_dot(ispm, cuda, dtype, n):
    noalloc, dot = _entry(ispm)
    code = 0 if dtype == "f32" else 1
    tdt = cuda.float32 if dtype == "f32" else cuda.float64
    gen = cuda.Generator(device="cuda").manual_seed(n)
    out = cuda.zeros(4, dtype=tdt, device="cuda")
    for call in range(2):  # two calls in a row, different data
        x = cuda.rand(n, dtype=tdt, device="cuda", generator=gen) - 0.5
        y = cuda.rand(n, dtype=tdt, device="cuda", generator=gen) - 0.5
        assert noalloc(code, x.data_ptr(), y.data_ptr(), out[0:1].data_ptr(), n, None) == 0, \
            ispm.lib_handle().ispm_last_error()
        assert dot(code, x.data_ptr(), y.data_ptr(), out[1:2].data_ptr(), n, None) == 0
        cuda.cuda.synchronize()
        a, b = out[0].item(), out[1].item()
        scale = (x.double() * y.double()).abs().sum().item()
        if dtype == "f64":
            assert abs(a - b) <= 1e-13 * scale, (call, a, b)
        else:
            assert a == b or abs(a - b) <= 1.2e-7 * max(abs(b), 1e-30), (call, a, b)


def test_noalloc_dot_rejects_bad_arguments(ispm, cuda):
    noalloc, _ = _entry(ispm)
    x = cuda.zeros(8, dtype=cuda.float64, device="cuda")
    assert noalloc(7, x.data_ptr(), x.data_ptr(), x.data_ptr(), 8, None) == ispm.ERR_INVALID
    assert noalloc(1, x.data_ptr(), x.data_ptr(), None, 8, None) == ispm.ERR_INVALID
    assert noalloc(1, x.data_ptr(), x.data_ptr(), x.data_ptr(), -1, None) == ispm.ERR_INVALID
