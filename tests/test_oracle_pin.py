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
@pytest.mark.parametrize("code", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("thermal", [False, True])
def test_decouple_pin(systems, name, code, thermal):
    """ABF, ANL, SEM, QI, True-IMPES and its second form, with and without the thermal variant
    (which only ANL / SEM / QI read), bit for bit against the reference library."""
    s = systems(name)
    a1, r1 = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, code, thermal=thermal)
    a2, r2 = oracle.ref_bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, code, thermal=thermal)
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


@pytest.mark.parametrize("name", ["small", "tiny3", "c0"])
@pytest.mark.parametrize("w,omega,direction", [(0.7, 0.9, 1), (1.0, 1.0, 1), (0.7, 0.9, -1)])
def test_hgs_relax_pin(systems, name, w, omega, direction):
    s = systems(name)
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    x0 = np.random.default_rng(1).standard_normal(s.n)
    got = oracle.hgs_relax(s.ia, s.ja, a, s.block_size, x0, b, w, omega, direction, 3)
    want = oracle.ref_hgs_relax(s.ia, s.ja, a, s.block_size, x0, b, w, omega, direction, 3)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("name", ["tiny", "small", "tiny3"])
def test_cpr_and_gmres_pin_live(systems, name):
    """Restatement vs the live reference: hierarchy, one CPR application, full solve."""
    s = systems(name)
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    R = oracle.RefCPR(s.ia, s.ja, a, s.block_size)
    O = oracle.OracleCPR(s.ia, s.ja, a, s.block_size)
    assert R.num_levels() == O.num_levels()
    for lev in range(R.num_levels()):
        ar, ao = R.level_matrix(lev, 0), O.level_matrix(lev, 0)
        for u, v in zip(ar[:3], ao[:3]):
            assert np.array_equal(u, v)
    r = np.random.default_rng(7).standard_normal(s.n)
    assert np.array_equal(R.apply(r), O.apply(r))
    ref = oracle.ref_gmres(s.ia, s.ja, s.a, s.block_size, s.b, decouple=1, tol=1e-6, max_iter=200)
    orc = oracle.gmres(s.ia, s.ja, a, s.block_size, b, tol=1e-6, max_iter=200, cpr=O)
    assert ref["iters"] == orc["iters"]
    assert np.array_equal(ref["x"], orc["x"])


@pytest.mark.parametrize("code", [2, 3, 4, 6])
def test_row_transform_consistent_rhs_keeps_solution(systems, code):
    """With the right-hand side transformed by the same row operation as the matrix, x_true still
    solves the decoupled system (the reference's aliased update does not keep it for ANL/SEM/QI)."""
    from jxpamg_all_b200.synth import bsr_matvec_np

    for name in ("tiny", "tiny3"):
        s = systems(name)
        a1, r1 = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, code, consistent_rhs=True)
        res = bsr_matvec_np(s.ia, s.ja, a1, s.block_size, s.x_true) - r1
        assert np.linalg.norm(res) <= 1e-10 * np.linalg.norm(r1)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("weights", [(0.7, 0.9), (1.0, 1.0)])
def test_hsgs_relax_pin(systems, name, weights):
    """jxf_ParBSRHSGSRelax (forward + backward pass; the work vector refreshed only in its first
    nb entries) against the reference, two calls in a row."""
    s = systems(name)
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    rng = np.random.default_rng(11)
    x0, w0 = rng.standard_normal(s.n), rng.standard_normal(s.n)
    x1, k1 = oracle.hsgs_relax(s.ia, s.ja, a, s.block_size, x0, b, w0, *weights, sweeps=2)
    x2, k2 = oracle.ref_hsgs_relax(s.ia, s.ja, a, s.block_size, x0, b, w0, *weights, sweeps=2)
    assert np.array_equal(x1, x2) and np.array_equal(k1, k2)


@pytest.mark.parametrize("name", NAMES)
def test_cpr_hsgs_stage2_pin(systems, name):
    """CPR with stage2_solver_type 3 (HSGS): two applications in a row and the full solve."""
    s = systems(name)
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    R = oracle.RefCPR(s.ia, s.ja, a, s.block_size, stage2_type=3)
    O = oracle.OracleCPR(s.ia, s.ja, a, s.block_size, stage2_type=3)
    r = np.random.default_rng(5).standard_normal(s.n)
    assert np.array_equal(R.apply(r), O.apply(r))
    assert np.array_equal(R.apply(b), O.apply(b))
    ref = oracle.ref_gmres(s.ia, s.ja, s.a, s.block_size, s.b, decouple=1, tol=1e-6, max_iter=200, stage2_type=3)
    orc = oracle.gmres(s.ia, s.ja, a, s.block_size, b, tol=1e-6, max_iter=200,
                       cpr=oracle.OracleCPR(s.ia, s.ja, a, s.block_size, stage2_type=3))
    assert ref["iters"] == orc["iters"]
