"""The oracle restatement against the golden fixtures made from the reference
(bit-exact: hierarchy patterns, CF splittings, CPR application, GMRES history
and solution).  Runs without the reference library."""
import numpy as np
import pytest

import oracle
from golden_util import CASES, load, sha


@pytest.mark.parametrize("name,decouple", CASES)
def test_oracle_matches_golden(systems, name, decouple):
    g = load(name, decouple)
    s = systems(name)
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, decouple)
    assert sha(a) == str(g["decoupled_a_sha"])
    assert sha(b) == str(g["decoupled_rhs_sha"])
    C = oracle.OracleCPR(s.ia, s.ja, a, s.block_size)
    assert C.num_levels() == int(g["num_levels"])
    for lev in range(C.num_levels()):
        ia, ja, av, m = C.level_matrix(lev, 0)
        assert sha(ia) == str(g[f"A{lev}_sha_ia"])
        assert sha(ja) == str(g[f"A{lev}_sha_ja"])
        assert np.abs(av).sum() == pytest.approx(float(g[f"A{lev}_sum_abs"]), rel=1e-13)
        if f"CF{lev}" in g:
            assert np.array_equal(C.level_cf(lev, len(ia) - 1), g[f"CF{lev}"].astype(np.int32))
            P = C.level_matrix(lev, 1)
            assert sha(P[0]) == str(g[f"P{lev}_sha_ia"])
            assert sha(P[1]) == str(g[f"P{lev}_sha_ja"])
            assert np.abs(P[2]).sum() == pytest.approx(float(g[f"P{lev}_sum_abs"]), rel=1e-13)
    assert np.array_equal(C.apply(g["cpr_r"]), g["cpr_z"])
    sol = oracle.gmres(s.ia, s.ja, a, s.block_size, b, tol=1e-6, max_iter=300, cpr=C)
    assert sol["iters"] == int(g["gmres_iters"])
    assert np.array_equal(sol["norms"], g["gmres_norms"])
    assert np.array_equal(sol["x"], g["gmres_x"])
