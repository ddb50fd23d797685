"""Block ILU(0) stage 2 on the GPU against the oracle (which is pinned to the
reference): factors, the tri-solve-14 application and the CPR application
with the BILU correction are bit-identical; the full solve converges."""
import numpy as np
import pytest

import oracle
from jxpamg_all_b200.solver import CprGmres

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["tiny", "small", "tiny3", "c0"])
@pytest.mark.parametrize("sweeps", [0, 3])
def test_bilu_factors_and_solve_bit_exact(systems, name, sweeps):
    s = systems(name)
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    G = CprGmres(decouple=1, stage2_solver_type=5, bilu_sweeps=sweeps).setup(s.ia, s.ja, s.a, s.block_size)
    F = oracle.bilu_setup(s.ia, s.ja, a, s.block_size, sweeps=sweeps)
    la, ua, dinv = G.bilu_factors()
    assert np.array_equal(la, F["la"]) and np.array_equal(ua, F["ua"]) and np.array_equal(dinv, F["dinv"])
    r = np.random.default_rng(4).standard_normal(s.n)
    assert np.array_equal(G.bilu_apply(r), oracle.bilu_solve(s.ia, s.ja, a, s.block_size, F, r))


@pytest.mark.parametrize("name", ["small", "c0"])
def test_cpr_with_bilu_stage_bit_exact(systems, name):
    s = systems(name)
    a, _ = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    G = CprGmres(decouple=1, stage2_solver_type=5).setup(s.ia, s.ja, s.a, s.block_size)
    O = oracle.OracleCPR(s.ia, s.ja, a, s.block_size, stage2_maxit=0)
    F = oracle.bilu_setup(s.ia, s.ja, a, s.block_size, sweeps=3)
    r = np.random.default_rng(8).standard_normal(s.n)
    assert np.array_equal(G.cpr_apply(r), oracle.cpr_bilu_apply(O, s.ia, s.ja, a, s.block_size, F, r))


@pytest.mark.parametrize("order,precision", [(0, 0), (1, 0), (1, 1)])
def test_bilu_stage_solve_converges(systems, order, precision):
    s = systems("c0")
    G = CprGmres(decouple=1, stage2_solver_type=5, smoother_order=order, coarse_exact=1 - order,
                 precision=precision, flexible=1 if precision else 0, max_iter=300).setup(
                     s.ia, s.ja, s.a, s.block_size)
    x, it, rel, conv = G.solve(s.b)
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    res = b - oracle.bsr_matvec(s.ia, s.ja, a, s.block_size, x)
    assert conv and np.linalg.norm(res) <= 1.05e-6 * np.linalg.norm(b)


# ---- exact BILU(0) with level-scheduled substitutions (bilu_exact 1) -------------------------------
@pytest.mark.parametrize("name", ["tiny", "small", "tiny3", "c0"])
def test_exact_bilu_levels_factors_and_solve_bit_exact(systems, name):
    """Levels computed on the device equal the oracle's longest-path levels; the exact factors and the
    level-scheduled solve are bit-identical to the oracle (itself pinned to the reference's sweeps and
    Jacobi solves at convergence, tests/test_bilu_oracle.py)."""
    s = systems(name)
    a, _ = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    G = CprGmres(decouple=1, stage2_solver_type=5, bilu_exact=1, bilu_ir_iters=3).setup(s.ia, s.ja, s.a,
                                                                                       s.block_size)
    lev_l, lev_u, nl, nu = G.bilu_levels()
    o_l, o_u, o_nl, o_nu = oracle.bilu_levels(s.ia, s.ja)
    assert (nl, nu) == (o_nl, o_nu)
    assert np.array_equal(lev_l, o_l) and np.array_equal(lev_u, o_u)
    F = oracle.bilu_setup_exact(s.ia, s.ja, a, s.block_size)
    la, ua, dinv = G.bilu_factors()
    assert np.array_equal(la, F["la"]) and np.array_equal(ua, F["ua"]) and np.array_equal(dinv, F["dinv"])
    r = np.random.default_rng(6).standard_normal(s.n)
    assert np.array_equal(G.bilu_apply(r), oracle.bilu_solve_exact(s.ia, s.ja, a, s.block_size, F, r, ir=3))
    G.close()


@pytest.mark.parametrize("name", ["c0", "tiny3"])
def test_exact_bilu_fp32_factors(systems, name):
    """The mixed path keeps the exact factors in FP32: its BILU application stays within FP32 rounding of
    the FP64 one."""
    s = systems(name)
    a, _ = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    G = CprGmres(decouple=1, stage2_solver_type=5, bilu_exact=1, smoother_order=1, coarse_exact=0, precision=1,
                 flexible=1).setup(s.ia, s.ja, s.a, s.block_size)
    F = oracle.bilu_setup_exact(s.ia, s.ja, a, s.block_size)
    r = np.random.default_rng(7).standard_normal(s.n)
    want = oracle.bilu_solve_exact(s.ia, s.ja, a, s.block_size, F, r)
    got = G.bilu_apply(r)
    assert np.linalg.norm(got - want) <= 1e-5 * np.linalg.norm(want)
    G.close()


@pytest.mark.parametrize("order,precision", [(0, 0), (1, 0), (1, 1)])
def test_exact_bilu_stage_solve_converges(systems, order, precision):
    s = systems("c0")
    G = CprGmres(decouple=1, stage2_solver_type=5, bilu_exact=1, smoother_order=order, coarse_exact=1 - order,
                 precision=precision, flexible=1 if precision else 0, max_iter=300).setup(
                     s.ia, s.ja, s.a, s.block_size)
    x, it, rel, conv = G.solve(s.b)
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    res = b - oracle.bsr_matvec(s.ia, s.ja, a, s.block_size, x)
    assert conv and np.linalg.norm(res) <= 1.05e-6 * np.linalg.norm(b)
    G.close()
