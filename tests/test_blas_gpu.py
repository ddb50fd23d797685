"""Device inner product (jxcpr_dot_dev) against a float64 numpy reference."""
import ctypes

import numpy as np
import pytest

from jxpamg_all_b200 import lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [0, 1, 7, 1000, 1 << 20, 2244000])
def test_dot_dev(n):
    from gpu_util import dev, ptr, stream

    rng = np.random.default_rng(n)
    x = rng.standard_normal(n)
    y = rng.standard_normal(n)
    xd, yd = dev(x), dev(y)
    out = np.zeros(1)
    lib.check(lib.load().jxcpr_dot_dev(n, ptr(xd), ptr(yd), out.ctypes.data_as(ctypes.c_void_p), stream()))
    want = float(np.dot(x, y))
    assert abs(out[0] - want) <= 1e-12 * max(1.0, np.abs(x).dot(np.abs(y)))
