"""jxcpr_dot_dev_noalloc: the inner product for callers that cannot allocate
device memory (applications whose own pool owns the GPU, loops that allow no
allocator call).

Checked through the C ABI against jxcpr_dot_dev on two calls in a row (the
second reuses the static scratch the first one left behind), plus the size
limit of that scratch.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from jxpamg_all_b200 import lib

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # same tolerance as tests/test_blas_gpu.py


def _dot(fn, xd, yd, n):
    from gpu_util import ptr, stream

    out = np.zeros(1)
    st = fn(n, ptr(xd), ptr(yd), out.ctypes.data_as(ctypes.c_void_p), stream())
    return st, float(out[0])


def test_noalloc_dot_matches_allocating_dot_twice():
    from gpu_util import dev

    so = lib.load()
    rng = np.random.default_rng(42)
    for n in (2244000, 3001):  # two calls in a row, the second smaller than the first
        x = rng.standard_normal(n)
        y = rng.standard_normal(n)
        xd, yd = dev(x), dev(y)
        st0, want = _dot(so.jxcpr_dot_dev, xd, yd, n)
        st1, got = _dot(so.jxcpr_dot_dev_noalloc, xd, yd, n)
        assert st0 == 0 and st1 == 0
        scale = max(1.0, float(np.abs(x).dot(np.abs(y))))
        assert abs(got - want) <= RTOL * scale
        assert abs(got - float(np.dot(x, y))) <= RTOL * scale


def test_noalloc_dot_leaves_free_memory_unchanged():
    """After the first call on the device (which loads the module and its static array),
    further calls take no device memory: cudaMemGetInfo's free bytes do not move."""
    import torch

    from gpu_util import dev

    so = lib.load()
    n = 1 << 20
    rng = np.random.default_rng(7)
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    xd, yd = dev(x), dev(y)
    st, _ = _dot(so.jxcpr_dot_dev_noalloc, xd, yd, 0)  # warm-up call, as the header asks
    assert st == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        st, got = _dot(so.jxcpr_dot_dev_noalloc, xd, yd, n)
        assert st == 0
        assert abs(got - float(np.dot(x, y))) <= RTOL * max(1.0, float(np.abs(x).dot(np.abs(y))))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_dot_rejects_sizes_beyond_scratch():
    from gpu_util import dev

    so = lib.load()
    xd = dev(np.zeros(4))
    limit = 4096 * 65536
    st, _ = _dot(so.jxcpr_dot_dev_noalloc, xd, xd, limit + 1)  # rejected before any device access
    assert st == 4
    assert b"static scratch limit" in so.jxcpr_last_error()
