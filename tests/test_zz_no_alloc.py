"""hpcgx_dot_noalloc: the dot product for callers that cannot allocate device
memory (code running inside another framework's memory pool, or latency-
critical loops where cudaMalloc/cudaFree would stall the device).

It is checked through the C ABI against the regular entry point hpcgx_dot
(which uses a problem's cudaMalloc'd scratch) on two calls in a row -- the
second call reuses the shared static scratch left by the first -- within the
1e-13 relative tolerance used for every dot product in these tests.  This
file is collected last, so that a run stopping at the first failure has run
everything else first; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_dot_noalloc_matches_dot_twice():
    from hpcg_b200 import Problem, _lib
    lib = _lib.lib()
    P = Problem(64, 64, 32)
    n = P.rows()
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) + 1.0
    y = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) - 0.5
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    for a, b in ((x, y), (x, x)):
        expected = P.dot(a, b)
        for call in range(2):
            out.fill_(float("nan"))
            rc = lib.hpcgx_dot_noalloc(n, _p(a), _p(b), _p(out), C.c_void_p(stream.cuda_stream))
            assert rc == 0, lib.hpcgx_last_error()
            torch.cuda.synchronize()
            got = out[0].item()
            assert abs(got / expected - 1.0) < 1e-13, (call, got, expected)
            assert torch.isnan(out[1])            # only the result slot is written


def test_dot_noalloc_sizes():
    from hpcg_b200 import _lib
    lib = _lib.lib()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    v = torch.ones(4099, dtype=torch.float64, device="cuda")
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.hpcgx_dot_noalloc(4099, _p(v), _p(v), _p(out), s) == 0
    torch.cuda.synchronize()
    assert out.item() == 4099.0
    assert lib.hpcgx_dot_noalloc(0, None, None, _p(out), s) == 0
    torch.cuda.synchronize()
    assert out.item() == 0.0
    # beyond the stated maximum: refused with a clear message, nothing launched
    assert lib.hpcgx_dot_noalloc(67108864 + 1, _p(v), _p(v), _p(out), s) == 1
    assert b"HPCGX_DOT_NOALLOC_MAX_N" in lib.hpcgx_last_error()
