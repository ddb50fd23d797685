"""Pins the oracle's C restatement to the reference library built from source.

Bit-exact agreement is required: both are plain IEEE double arithmetic in the
same order (see the citations in oracle/orc_bsr.c).
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.ref

NAMES = ["tiny", "small", "tiny3", "c0"]


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-1.0, 1.0), (2.5, -0.75), (0.0, 3.0), (1.0, 1.0)])
def test_bsr_matvec_pin(systems, name, alpha, beta):
    s = systems(name)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(s.n)
    y0 = rng.standard_normal(s.n)
    got = oracle.bsr_matvec(s.ia, s.ja, s.a, s.block_size, x, alpha, y0, beta)
    want = oracle.ref_bsr_matvec(s.ia, s.ja, s.a, s.block_size, x, alpha, y0, beta)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("code", [1, 5])
def test_decouple_pin(systems, name, code):
    s = systems(name)
    a1, r1 = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, code)
    a2, r2 = oracle.ref_bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, code)
    assert np.array_equal(a1, a2)
    assert np.array_equal(r1, r2)


def test_abf_consistent_rhs_keeps_solution(systems):
    """The corrected right-hand-side update preserves the solution; the reference one does not."""
    from jxpamg_all_b200.synth import bsr_matvec_np

    s = systems("tiny")
    a1, r1 = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1, consistent_rhs=True)
    res = bsr_matvec_np(s.ia, s.ja, a1, s.block_size, s.x_true) - r1
    assert np.linalg.norm(res) <= 1e-10 * np.linalg.norm(r1)
    a2, r2 = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    assert np.array_equal(a1, a2)
    assert not np.allclose(r1, r2)
