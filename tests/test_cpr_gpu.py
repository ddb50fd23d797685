"""CPR-GMRES on the GPU against the oracle (restatement pinned to the reference).

In the exact-order mode (smoother_order 0, coarse_exact 1) everything the
preconditioner computes is bit-identical to the oracle: decoupled matrix, AMG
hierarchy (C/F splittings, P, coarse operators), V-cycle and CPR application.
GMRES differs only by the summation order of its device dot products, so the
full solve is compared with tolerances: equal iteration counts and residual
histories within 1e-9 relative.
"""
import numpy as np
import pytest

import oracle
from jxpamg_all_b200.solver import CprGmres

pytestmark = pytest.mark.gpu

CASES = [("tiny", 1), ("small", 1), ("small", 5), ("c0", 1), ("c0", 5), ("tiny3", 1), ("tiny3", 5)]


def build(s, decouple, **opt):
    return CprGmres(decouple=decouple, **opt).setup(s.ia, s.ja, s.a, s.block_size)


@pytest.mark.parametrize("name,decouple", CASES)
def test_hierarchy_bit_exact(systems, name, decouple):
    s = systems(name)
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, decouple)
    G = build(s, decouple)
    assert np.array_equal(G.decoupled_values(s.nnzb), a)
    O = oracle.OracleCPR(s.ia, s.ja, a, s.block_size)
    assert G.num_levels() == O.num_levels()
    for lev in range(O.num_levels()):
        go, oo = G.level_matrix(lev, 0), O.level_matrix(lev, 0)
        for u, v in zip(go[:3], oo[:3]):
            assert np.array_equal(u, v), f"A{lev}"
        if lev < O.num_levels() - 1:
            n = len(oo[0]) - 1
            assert np.array_equal(G.level_cf(lev, n), O.level_cf(lev, n)), f"CF{lev}"
            gp, op = G.level_matrix(lev, 1), O.level_matrix(lev, 1)
            for u, v in zip(gp[:3], op[:3]):
                assert np.array_equal(u, v), f"P{lev}"


@pytest.mark.parametrize("name,decouple", CASES)
def test_vcycle_and_cpr_bit_exact(systems, name, decouple):
    s = systems(name)
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, decouple)
    G = build(s, decouple)
    O = oracle.OracleCPR(s.ia, s.ja, a, s.block_size)
    rng = np.random.default_rng(11)
    rp = rng.standard_normal(s.num_block_rows)
    assert np.array_equal(G.vcycle(rp), O.vcycle(rp))
    r = rng.standard_normal(s.n)
    assert np.array_equal(G.cpr_apply(r), O.apply(r))


@pytest.mark.parametrize("name,decouple", CASES)
def test_solve_matches_oracle(systems, name, decouple):
    s = systems(name)
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, decouple)
    O = oracle.OracleCPR(s.ia, s.ja, a, s.block_size)
    ref = oracle.gmres(s.ia, s.ja, a, s.block_size, b, tol=1e-6, max_iter=300, cpr=O)
    G = build(s, decouple, max_iter=300)
    x, it, rel, conv = G.solve(s.b)
    assert conv and rel <= 1e-6
    assert it == ref["iters"]
    # only the dot products' summation order differs: histories agree to ~1e-9
    assert np.allclose(G.norms(), ref["norms"], rtol=1e-7, atol=0)
    # x agrees with the oracle's solution far below the solver tolerance
    assert np.linalg.norm(x - ref["x"]) <= 1e-8 * np.linalg.norm(ref["x"])
    # true residual of the decoupled system
    res = oracle.bsr_matvec(s.ia, s.ja, a, s.block_size, x, -1.0, b, 1.0)
    assert np.linalg.norm(res) <= 1e-6 * np.linalg.norm(b) * (1 + 1e-9)


def test_solve_golden(systems):
    """Against the fixtures made by the reference library itself."""
    from golden_util import load

    for name, dec in [("c0", 1), ("c0", 5)]:
        g = load(name, dec)
        s = systems(name)
        G = build(s, dec, max_iter=300)
        x, it, rel, conv = G.solve(s.b)
        assert it == int(g["gmres_iters"])
        assert np.allclose(G.norms(), g["gmres_norms"], rtol=1e-7, atol=0)
        assert np.linalg.norm(x - g["gmres_x"]) <= 1e-8 * np.linalg.norm(g["gmres_x"])


def test_multicolor_mode_converges(systems):
    """The throughput mode (multicolour Gauss-Seidel on level 0, l1-Jacobi on dense
    coarse levels) is a different smoother; it must still converge to the
    tolerance with an iteration count within +-10 % of the reference's."""
    s = systems("c0")
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    O = oracle.OracleCPR(s.ia, s.ja, a, s.block_size)
    ref = oracle.gmres(s.ia, s.ja, a, s.block_size, b, tol=1e-6, max_iter=300, cpr=O)
    G = build(s, 1, max_iter=300, smoother_order=1, coarse_exact=0)
    x, it, rel, conv = G.solve(s.b)
    assert conv and rel <= 1e-6
    assert abs(it - ref["iters"]) <= 0.10 * ref["iters"]
    res = oracle.bsr_matvec(s.ia, s.ja, a, s.block_size, x, -1.0, b, 1.0)
    assert np.linalg.norm(res) <= 1e-6 * np.linalg.norm(b) * (1 + 1e-9)
