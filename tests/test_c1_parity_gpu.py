"""Parity on the benchmarked workload: the 1,122,000-cell channelised system
(60x220x85, 2x2 BSR, 7.78M blocks, seed 1, ABF decoupling, CPR-GMRES(30) to
FP64 rel-res 1e-6) against the fixture the reference library wrote
(tests/golden/c1_dec1.npz, made by tests/golden/make_golden.py c1 with one
OpenMP thread: 6 AMG levels, 51 GMRES iterations).

* exact-order mode: decoupled matrix, every level's C/F splitting and A_l / P_l
  patterns equal (SHA-256), the same 51 iterations, residual history within
  1e-7 and the solution within 1e-8 relative (on the fixture's 65,536 sampled
  entries and in norm);
* throughput path with a one-range coarsening first pass: the same hierarchy;
* the plain FP64 throughput path: iterations within +-10 % of the reference's;
  the measured mixed-precision path (the benchmark's options): at most 10 %
  more; both a true FP64 residual below 1e-6 and the solution's distance from
  the reference's FP64 solution stated.
"""
import numpy as np
import pytest

import oracle
from golden_util import load, sha
from jxpamg_all_b200.solver import CprGmres

pytestmark = pytest.mark.gpu

REF_ITERS_TOL = 0.10  # iteration counts within +-10 % of the reference's


@pytest.fixture(scope="module")
def c1(systems):
    s = systems("c1")
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    return s, a, b, load("c1", 1)


def _check_hierarchy(G, g, s):
    assert G.num_levels() == int(g["num_levels"])
    for lev in range(G.num_levels()):
        ia, ja, av, m = G.level_matrix(lev, 0)
        n = len(ia) - 1
        assert n == int(g[f"A{lev}_n"]), f"A{lev} rows"
        assert sha(ia) == str(g[f"A{lev}_sha_ia"]), f"A{lev} ia"
        assert sha(ja) == str(g[f"A{lev}_sha_ja"]), f"A{lev} ja"
        assert np.abs(av).sum() == pytest.approx(float(g[f"A{lev}_sum_abs"]), rel=1e-12)
        if f"CF{lev}_sha" in g:
            cf = G.level_cf(lev, n)
            assert sha(cf.astype(np.int8)) == str(g[f"CF{lev}_sha"]), f"CF{lev}"
            P = G.level_matrix(lev, 1)
            assert sha(P[0]) == str(g[f"P{lev}_sha_ia"]), f"P{lev} ia"
            assert sha(P[1]) == str(g[f"P{lev}_sha_ja"]), f"P{lev} ja"
            assert np.abs(P[2]).sum() == pytest.approx(float(g[f"P{lev}_sum_abs"]), rel=1e-12)


def _x_error(x, g):
    """Relative distance from the reference's FP64 solution on the sampled entries."""
    idx = g["x_sample_idx"]
    ref = g["x_sample"]
    return float(np.linalg.norm(x[idx] - ref) / np.linalg.norm(ref))


def _true_rel_res(s, a, b, x):
    r = oracle.bsr_matvec(s.ia, s.ja, a, s.block_size, x, -1.0, b, 1.0)
    return float(np.linalg.norm(r) / np.linalg.norm(b))


def test_c1_exact_mode_matches_reference(c1):
    s, a, b, g = c1
    G = CprGmres(decouple=1, smoother_order=0, coarse_exact=1, max_iter=300).setup(s.ia, s.ja, s.a,
                                                                                   s.block_size)
    assert sha(G.decoupled_values(s.nnzb)) == str(g["decoupled_a_sha"])
    _check_hierarchy(G, g, s)
    x, it, rel, conv = G.solve(s.b)
    assert conv and rel <= 1e-6
    assert it == int(g["gmres_iters"])
    assert np.allclose(G.norms(), g["gmres_norms"], rtol=1e-7, atol=0)
    assert _x_error(x, g) <= 1e-8
    assert abs(np.linalg.norm(x) - float(g["x_norm2"])) <= 1e-8 * float(g["x_norm2"])
    assert _true_rel_res(s, a, b, x) <= 1e-6 * (1 + 1e-9)
    G.close()


def test_c1_throughput_hierarchy_one_range_matches_reference(c1):
    """The throughput path builds the same hierarchy as the reference when its coarsening's
    first pass runs over the whole level (rs_range_rows 0)."""
    s, a, b, g = c1
    G = CprGmres(decouple=1, smoother_order=1, coarse_exact=0, precision=0, fast_smoother=0,
                 rs_range_rows=0).setup(s.ia, s.ja, s.a, s.block_size)
    _check_hierarchy(G, g, s)
    G.close()


def _fast_solve(c1, opts, fewer_ok=False):
    s, a, b, g = c1
    G = CprGmres(**opts).setup(s.ia, s.ja, s.a, s.block_size)
    x, it, rel, conv = G.solve(s.b)
    G.close()
    ref_it = int(g["gmres_iters"])
    assert conv and rel <= 1e-6
    if fewer_ok:
        assert it <= (1 + REF_ITERS_TOL) * ref_it, f"{it} iterations vs the reference's {ref_it}"
    else:
        assert abs(it - ref_it) <= REF_ITERS_TOL * ref_it, f"{it} iterations vs the reference's {ref_it}"
    assert _true_rel_res(s, a, b, x) <= 1e-6 * (1 + 1e-9)
    return it, _x_error(x, g)


def test_c1_plain_fp64_throughput_path(c1):
    """The reference's method (weights 0.7 / 0.9, FP64) in the throughput orderings: within +-10 %
    of the reference's iterations (the chunk-ordered stage 2 keeps the natural sweep's coupling)."""
    import bench

    it, err = _fast_solve(c1, bench.PLAIN_OPTS)
    # same method, other smoother orderings: the solutions differ by what a 1e-6 residual leaves
    assert err <= 1e-2, err
    print(f"plain FP64 throughput path: {it} iterations, x vs the reference's FP64 solution {err:.2e}")


def test_c1_mixed_measured_path(c1):
    """The measured path changes the method on purpose (FP32 storage, learned strength thresholds and
    Chebyshev intervals, the mixed driver's stage-2 weights): at most 10 % more iterations than the
    reference (fewer are allowed), the same true FP64 residual, and its distance from the
    reference's FP64 solution stated."""
    import bench

    it, err = _fast_solve(c1, bench.SOLVER_OPTS, fewer_ok=True)
    assert err <= 1e-2, err
    print(f"mixed + learned path: {it} iterations, x vs the reference's FP64 solution {err:.2e}")


def test_c1_bf16_coarse_levels_path(c1):
    """The BF16 form (coarse levels in BF16 with per-block scales, FP32 level 0 and stage 2, FP64 GMRES and
    coarsest solve): converges to the true FP64 residual; its iterations and its distance from the
    reference's FP64 solution are stated."""
    import bench

    s, a, b, g = c1
    G = CprGmres(**dict(bench.SOLVER_OPTS, precision=2)).setup(s.ia, s.ja, s.a, s.block_size)
    x, it, rel, conv = G.solve(s.b)
    G.close()
    assert conv and rel <= 1e-6
    assert _true_rel_res(s, a, b, x) <= 1e-6 * (1 + 1e-9)
    err = _x_error(x, g)
    assert err <= 1e-2, err
    print(f"BF16 coarse levels: {it} iterations (reference {int(g['gmres_iters'])}), x vs the reference's FP64 "
          f"solution {err:.2e}")
