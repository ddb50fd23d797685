"""The coarsest-level inverse of the fast path (blocked Gauss-Jordan without pivoting, one cooperative
kernel with FP64 tensor-core updates) against FP64 references: numpy's inverse on dense matrices of
sizes around the 32-wide blocking, and the exact path's substitution in jxf_gselim's order on the
coarsest operator of real hierarchies (through one V-cycle)."""
import ctypes

import numpy as np
import pytest

from jxpamg_all_b200 import lib
from jxpamg_all_b200.solver import CprGmres

pytestmark = pytest.mark.gpu


def dense_inverse(a):
    import torch

    from gpu_util import dev, stream

    so = lib.load()
    n = a.shape[0]
    d_a = dev(a)
    d_x = torch.empty((n, n), dtype=torch.float64, device="cuda")
    st = so.jxcpr_dense_inverse_dev(n, d_a.data_ptr(), d_x.data_ptr(), ctypes.c_void_p(stream()))
    torch.cuda.synchronize()
    return st, d_x.cpu().numpy()


def coarse_like(n, seed):
    """Non-symmetric, diagonally dominant, M-matrix-like (a coarse pressure operator's shape)."""
    rng = np.random.default_rng(seed)
    a = -np.abs(rng.standard_normal((n, n))) * (rng.random((n, n)) < min(1.0, 40.0 / n))
    np.fill_diagonal(a, 0.0)
    np.fill_diagonal(a, -a.sum(axis=1) + 0.05 + rng.random(n))
    return a


@pytest.mark.parametrize("n", [1, 2, 31, 32, 33, 100, 420, 632, 1000, 2000])
def test_dense_inverse_matches_fp64(n):
    a = coarse_like(n, n)
    st, x = dense_inverse(a)
    assert st == 0, lib.load().jxcpr_last_error()
    want = np.linalg.inv(a)
    assert np.linalg.norm(x - want) <= 1e-12 * np.linalg.cond(a) * np.linalg.norm(want)
    assert np.linalg.norm(a @ x - np.eye(n)) <= 1e-11 * np.sqrt(n)


def test_dense_inverse_zero_pivot_is_reported():
    a = coarse_like(64, 3)
    a[5, 5] = 0.0
    a[5, :] = 0.0  # an empty row: the elimination meets a zero pivot
    st, _ = dense_inverse(a)
    assert st == 4
    assert b"zero pivot" in lib.load().jxcpr_last_error()


@pytest.mark.parametrize("name", ["small", "c0", "tiny3"])
def test_vcycle_with_inverse_matches_substitution(systems, name):
    """Exact-order V-cycle with the coarse inverse (coarse_exact 0) against the one with the
    reference-order substitution (coarse_exact 1): only the coarse solve's rounding differs."""
    s = systems(name)
    rp = np.random.default_rng(5).standard_normal(s.num_block_rows)
    out = []
    for ce in (1, 0):
        G = CprGmres(decouple=1, smoother_order=0, coarse_exact=ce).setup(s.ia, s.ja, s.a, s.block_size)
        out.append(G.vcycle(rp))
        G.close()
    assert np.linalg.norm(out[1] - out[0]) <= 1e-10 * np.linalg.norm(out[0])
