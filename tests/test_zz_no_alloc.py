"""The allocation-free dot product, fb_dot_f64_noalloc, checked against fb_dot_f64.

Some callers of this library cannot call cudaMalloc when they need a reduction: their device
memory belongs to an external allocator, or their process forbids allocation after start-up.
For them the library offers a dot product whose scratch is a fixed device array compiled into
the library, so no call allocates or frees memory. This file calls both entry points through
the C-ABI on the same inputs and requires agreement within the tolerance the other FP64
reduction tests use. It makes two calls in a row, so the second call runs on the scratch that
the first one left behind. It also checks that a size above the fixed limit is refused with
FB_ERR_TOO_LARGE. The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # same bound as the FP64 dot checks of tests/test_gpu_ops.py


def _dot(lib, name, x, y):
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = getattr(lib, name)(x.data_ptr(), y.data_ptr(), x.numel(), out.data_ptr(), stream)
    assert rc == 0, f"{name} returned status {rc}"
    torch.cuda.current_stream().synchronize()
    return float(out.item())


def test_noalloc_dot_matches_allocating_dot_twice():
    from feat3_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(7)
    for n in (3_000_001, 4_097):  # the second call reuses the scratch left by the first
        x = torch.tensor(rng.standard_normal(n), device="cuda")
        y = torch.tensor(rng.standard_normal(n) + 0.5, device="cuda")
        ref = _dot(lib, "fb_dot_f64", x, y)
        got = _dot(lib, "fb_dot_f64_noalloc", x, y)
        assert got == pytest.approx(ref, rel=RTOL, abs=RTOL * float(torch.sum(torch.abs(x * y))))
        assert got == pytest.approx(float(np.dot(x.cpu().numpy(), y.cpu().numpy())), rel=1e-10)


def test_noalloc_dot_refuses_sizes_beyond_its_scratch():
    from feat3_b200 import _lib
    lib = _lib.load()
    x = torch.zeros(16, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    max_n = 4096 * 16384  # FB_NOALLOC_DOT_MAX_N
    # the size check happens before any device work, so the short buffers are never read
    rc = lib.fb_dot_f64_noalloc(x.data_ptr(), x.data_ptr(), max_n + 1, out.data_ptr(), None)
    assert rc == _lib.FB_ERR_TOO_LARGE
    assert lib.fb_dot_f64_noalloc(None, None, 10, out.data_ptr(), None) == _lib.FB_ERR_INVALID
    assert _dot(lib, "fb_dot_f64_noalloc", x, x) == 0.0
    assert ctypes.c_int(rc).value == 6
