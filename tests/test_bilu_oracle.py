"""Block ILU(0) restatement (oracle/orc_bilu.c) pinned to the reference's own
jxf_BILUSetup (type 3) + jxf_BILUSolve (tri-solve 14), compiled from its
sources: factors and solution bit-identical on every system and sweep count."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.ref


@pytest.mark.parametrize("name", ["tiny", "small", "tiny3", "c0"])
@pytest.mark.parametrize("sweeps", [0, 1, 3])
def test_bilu_restatement_matches_reference(systems, name, sweeps):
    s = systems(name)
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    F = oracle.bilu_setup(s.ia, s.ja, a, s.block_size, sweeps=sweeps)
    u = oracle.bilu_solve(s.ia, s.ja, a, s.block_size, F, b)
    ur, la, ua, dinv = oracle.ref_bilu(s.ia, s.ja, a, s.block_size, b, sweeps=sweeps)
    assert np.array_equal(F["la"], la)
    assert np.array_equal(F["ua"], ua)
    assert np.array_equal(F["dinv"], dinv)
    assert np.array_equal(u, ur)


def test_bilu_converges_to_ilu0_fixed_point(systems):
    """Many sweeps reach the exact BILU(0): A = (I+L)(D+U) on the pattern of A."""
    s = systems("small")
    a, _ = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    F40 = oracle.bilu_setup(s.ia, s.ja, a, s.block_size, sweeps=40)
    F41 = oracle.bilu_setup(s.ia, s.ja, a, s.block_size, sweeps=41)
    assert np.allclose(F40["la"], F41["la"], rtol=1e-12, atol=1e-14)
    assert np.allclose(F40["ua"], F41["ua"], rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("name", ["tiny", "small", "tiny3", "c0"])
def test_exact_bilu_matches_reference_at_convergence(systems, name):
    """The exact factors and level-ordered solves of the restatement equal the reference's FGPBILU
    sweeps and Jacobi triangular solves once their counts exceed the DAG levels: bit for bit."""
    s = systems(name)
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    lev_l, lev_u, nl, nu = oracle.bilu_levels(s.ia, s.ja)
    F = oracle.bilu_setup_exact(s.ia, s.ja, a, s.block_size)
    u = oracle.bilu_solve_exact(s.ia, s.ja, a, s.block_size, F, b, ir=3)
    ur, la, ua, dinv = oracle.ref_bilu(s.ia, s.ja, a, s.block_size, b, sweeps=max(nl, nu) + 2, ir=3,
                                       lower=nl + 1, upper=nu + 1)
    assert np.array_equal(F["la"], la)
    assert np.array_equal(F["ua"], ua)
    assert np.array_equal(F["dinv"], dinv)
    assert np.array_equal(u, ur)
