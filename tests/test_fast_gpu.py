"""The throughput / mixed-precision path (smoother_order 1) on the GPU.

Its orderings differ from the reference (multicolour Gauss-Seidel, l1-Jacobi or
Chebyshev on dense levels, FP32/BF16 storage), so parity is checked through
what the method guarantees: GMRES reaches the tolerance on the TRUE residual
of the decoupled system (recomputed here on the CPU with the oracle), the
hierarchy is the exact path's one for the default thresholds, and options that
must not change results (CUDA-graph replay) do not.
"""
import numpy as np
import pytest

import oracle
from jxpamg_all_b200.solver import CprGmres
from jxpamg_all_b200 import synth

pytestmark = pytest.mark.gpu

BASE = dict(decouple=1, max_iter=400, smoother_order=1, coarse_exact=0)


def true_rel(s, x, decouple=1):
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, decouple)
    r = b - synth.bsr_matvec_np(s.ia, s.ja, a, s.block_size, x)
    return np.linalg.norm(r) / np.linalg.norm(b)


def solve(s, **opt):
    G = CprGmres(**dict(BASE, **opt)).setup(s.ia, s.ja, s.a, s.block_size)
    x, it, rel, conv = G.solve(s.b)
    return G, x, it, rel, conv


VARIANTS = [
    dict(precision=0, fast_smoother=0),
    dict(precision=0, fast_smoother=1),
    dict(precision=0, fast_smoother=3),
    dict(precision=1, fast_smoother=0, flexible=1),
    dict(precision=1, fast_smoother=1, flexible=1),
    dict(precision=2, fast_smoother=1, flexible=1),
    dict(precision=1, fast_smoother=2, flexible=1),
    dict(precision=2, fast_smoother=2, flexible=1),
    dict(precision=0, fast_smoother=0, orthog=1),
    dict(precision=1, fast_smoother=1, flexible=1, autotune=0, graphs=0),
    dict(precision=0, fast_smoother=1, strong_threshold=0.5, strong_threshold_coarse=0.7),
    # the reference's hybrid form: FP32 stage 1, FP64 stage 2 polish with weights 1.0 / 0.8
    dict(precision=3, fast_smoother=0, flexible=1, stage2_relax_weight=1.0, stage2_omega=0.8),
    dict(precision=3, fast_smoother=1, flexible=1),
]


@pytest.mark.parametrize("name", ["small", "c0", "tiny3", "slab_small"])
@pytest.mark.parametrize("opt", VARIANTS, ids=lambda o: "-".join(f"{k}{v}" for k, v in o.items()))
def test_variants_reach_true_residual(systems, name, opt):
    s = systems(name) if name != "slab_small" else synth.reservoir_system(30, 110, 12, seed=21, phases=2,
                                                                         channelised_layers=7)
    G, x, it, rel, conv = solve(s, **opt)
    assert conv, (it, rel)
    assert true_rel(s, x) <= 1.05e-6
    G.close()


def test_graph_replay_is_identical(systems):
    s = systems("c0")
    _, x1, it1, _, _ = solve(s, precision=1, fast_smoother=1, flexible=1, graphs=1, autotune=0)
    _, x2, it2, _, _ = solve(s, precision=1, fast_smoother=1, flexible=1, graphs=0, autotune=0)
    assert it1 == it2 and np.array_equal(x1, x2)


def test_mixed_solution_close_to_fp64(systems):
    s = systems("c0")
    _, x64, _, _, _ = solve(s, precision=0, fast_smoother=0)
    for p in (1, 2):
        _, xm, _, _, _ = solve(s, precision=p, fast_smoother=1, flexible=1)
        assert np.linalg.norm(xm - x64) <= 1e-3 * np.linalg.norm(x64)


def test_level_storage_and_smoothers(systems):
    s = systems("c0")
    G, *_ = solve(s, precision=2, fast_smoother=1, flexible=1, bf16_level=1)
    L = G.num_levels()
    for lev in range(L - 1):
        info = G.level_info(lev)
        assert info["storage"] == (1 if lev == 0 else 2)
        assert info["smoother"] in (1, 3)
        if info["smoother"] == 3:
            lo, hi = info["interval"]
            c0, c1, c2 = info["cheb"]
            t = np.linspace(lo, hi, 101)
            q = 1 - t * (c0 + c1 * t + c2 * t * t)  # error polynomial of one application
            sg = (hi + lo) / (hi - lo)
            assert np.max(np.abs(q)) <= 1.0 / (4 * sg ** 3 - 3 * sg) * (1 + 1e-9)
    assert G.level_info(L - 1)["smoother"] == 0


def test_default_threshold_hierarchy_matches_exact_path(systems):
    """The fast path coarsens with the reference's rules: same hierarchy as the exact path."""
    s = systems("small")
    E = CprGmres(decouple=1).setup(s.ia, s.ja, s.a, s.block_size)
    F, *_ = solve(s, precision=1, fast_smoother=1, flexible=1)
    assert E.num_levels() == F.num_levels()
    for lev in range(E.num_levels()):
        for u, v in zip(E.level_matrix(lev)[:3], F.level_matrix(lev)[:3]):
            assert np.array_equal(u, v)


@pytest.mark.parametrize("rows", [1000, 2000, 3000])
def test_first_pass_on_row_ranges_matches_oracle(systems, rows):
    """rs_range_rows: the coarsening's first pass runs on row ranges (each on its own diagonal
    block of the strength pattern, on host threads); every level's C/F splitting equals the
    oracle's ranged HMIS on that level's operator, and the solve still converges."""
    s = systems("c0")
    F, x, it, rel, conv = solve(s, precision=1, fast_smoother=1, flexible=1, rs_range_rows=rows)
    G, x0, it0, rel0, conv0 = solve(s, precision=1, fast_smoother=1, flexible=1, rs_range_rows=0)
    ranged = 0
    for lev in range(F.num_levels() - 1):
        ia, ja, a = F.level_matrix(lev)[:3]
        n = len(ia) - 1
        ranged += n >= 2 * rows
        assert np.array_equal(F.level_cf(lev, n), oracle.hmis_cf(ia, ja, a, range_rows=rows)), lev
    assert ranged >= 1
    assert conv and conv0 and abs(it - it0) <= max(2, it0 // 10), (it, it0)
    assert true_rel(s, x) <= 1.05e-6
    F.close()
    G.close()


def test_row_ranges_leave_small_levels_whole(systems):
    """Levels with fewer than two ranges' rows (and the exact order always) coarsen in one pass."""
    s = systems("small")
    E = CprGmres(decouple=1, rs_range_rows=100).setup(s.ia, s.ja, s.a, s.block_size)
    O = oracle.OracleCPR(s.ia, s.ja, oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)[0], s.block_size)
    n = len(O.level_matrix(0, 0)[0]) - 1
    assert np.array_equal(E.level_cf(0, n), O.level_cf(0, n))
    F, *_ = solve(s, precision=1, fast_smoother=1, flexible=1, rs_range_rows=n)
    assert np.array_equal(F.level_cf(0, n), O.level_cf(0, n))
    for G in (E, F):
        G.close()


def test_stage2_native_and_autotune_report(systems):
    from jxpamg_all_b200 import lib

    s = systems("c0")
    G, *_ = solve(s, precision=1, fast_smoother=1, flexible=1)
    lib.check(lib.load().jxcpr_solver_stage2_native(G.h, 2))
    rep = G.setup_report()
    assert "tuned stage2" in rep and "tuned A0" in rep


def test_hybrid_stage2_is_fp64(systems):
    """precision 3 runs stage 2 in FP64 on the FP64 matrix: with the stage-1 AMG switched off
    (stage1_maxit 0 is not allowed, so compare stage-2 sweeps directly) one sweep from the same
    iterate matches the FP64 fast path's sweep to FP64 rounding."""
    s = systems("c0")
    rng = np.random.default_rng(4)
    r = rng.standard_normal(s.n)
    z0 = rng.standard_normal(s.n)
    out = []
    for p in (0, 3):
        G, *_ = solve(s, precision=p, fast_smoother=0, flexible=1, autotune=0)
        out.append(G.stage2_sweep(r, z0))
        G.close()
    assert np.linalg.norm(out[0] - out[1]) <= 1e-12 * np.linalg.norm(out[0])


def _greedy_classes(ia, ja, n):
    """Colour classes of the fast path's level-0 schedule: greedy colouring of the symmetrised
    pattern in natural order."""
    nbrs = [set() for _ in range(n)]
    for i in range(n):
        for k in range(ia[i], ia[i + 1]):
            j = int(ja[k])
            if j != i:
                nbrs[i].add(j)
                nbrs[j].add(i)
    color = [-1] * n
    for i in range(n):
        used = {color[j] for j in nbrs[i] if color[j] >= 0}
        c = 0
        while c in used:
            c += 1
        color[i] = c
    return np.array(color)


@pytest.mark.parametrize("name", ["small", "c0", "tiny3"])
@pytest.mark.parametrize("chunk", [4, 8, 16])
@pytest.mark.parametrize("weights", [(0.7, 0.9), (1.0, 1.0), (1.0, 0.8)], ids=["ref", "plain", "mixed"])
def test_stage2_sweep_matches_chunk_ordered_hgs(systems, name, chunk, weights):
    """One FP64 stage-2 sweep of the fast path in chunk order (the default) against the oracle's
    restatement of the reference's weighted block update visited in the same order
    (oracle.hgs_relax_chunked); only the summation order of each row differs."""
    s = systems(name)
    bs = s.block_size
    a_dec, _ = oracle.bsr_decouple(s.ia, s.ja, s.a, bs, s.b, 1)
    w, om = weights
    G, *_ = solve(s, precision=0, fast_smoother=0, stage2_chunk=chunk, stage2_relax_weight=w, stage2_omega=om)
    rng = np.random.default_rng(9)
    r = rng.standard_normal(s.n)
    z0 = rng.standard_normal(s.n)
    got = G.stage2_sweep(r, z0)
    G.close()
    want = oracle.hgs_relax_chunked(s.ia, s.ja, a_dec, bs, z0, r, chunk, w=w, omega=om)
    assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want)


@pytest.mark.parametrize("name", ["c0", "tiny3"])
def test_stage2_sweep_fp32_chunk_order(systems, name):
    """The mixed path's FP32 stage-2 sweep in chunk order against the FP64 restatement (FP32 rounding)."""
    s = systems(name)
    bs = s.block_size
    a_dec, _ = oracle.bsr_decouple(s.ia, s.ja, s.a, bs, s.b, 1)
    G, *_ = solve(s, precision=1, fast_smoother=0, flexible=1, stage2_chunk=4)
    rng = np.random.default_rng(10)
    r = rng.standard_normal(s.n)
    z0 = rng.standard_normal(s.n)
    got = G.stage2_sweep(r, z0)
    G.close()
    want = oracle.hgs_relax_chunked(s.ia, s.ja, a_dec, bs, z0, r, 4)
    assert np.linalg.norm(got - want) <= 1e-5 * np.linalg.norm(want)


@pytest.mark.parametrize("name", ["small", "c0", "tiny3"])
@pytest.mark.parametrize("opt", [dict(autotune=0), dict(autotune=1)], ids=["heuristic", "tuned"])
def test_stage2_sweep_matches_colour_ordered_hgs(systems, name, opt):
    """One FP64 stage-2 sweep of the fast path in the level-0 colour order (stage2_chunk 0: colour
    classes in order, no start-of-sweep copy) against a direct restatement of the weighted block
    Gauss-Seidel update with vt = the iterate at the sweep start:
    x_i <- (1 - w om) vt_i + w D_i^-1 (om b_i - sum_j A_ij (x_j - (1 - om) vt_j))."""
    s = systems(name)
    bs = s.block_size
    a_dec, _ = oracle.bsr_decouple(s.ia, s.ja, s.a, bs, s.b, 1)
    G, *_ = solve(s, precision=0, fast_smoother=0, stage2_chunk=0, **opt)
    rng = np.random.default_rng(8)
    r = rng.standard_normal(s.n)
    z0 = rng.standard_normal(s.n)
    got = G.stage2_sweep(r, z0)
    G.close()
    nb = s.num_block_rows
    A = a_dec.reshape(-1, bs, bs)
    color = _greedy_classes(s.ia, s.ja, nb)
    w, om = 0.7, 0.9
    vt = z0.reshape(nb, bs).copy()
    x = vt.copy()
    R = r.reshape(nb, bs)
    for c in range(color.max() + 1):
        for i in np.nonzero(color == c)[0]:
            acc = np.zeros(bs)
            for k in range(s.ia[i] + 1, s.ia[i + 1]):
                j = s.ja[k]
                acc += A[k] @ (x[j] - (1 - om) * vt[j])
            out = np.linalg.solve(A[s.ia[i]], om * R[i] - acc)
            x[i] = (1 - w * om) * vt[i] + w * out
    want = x.reshape(-1)
    assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want)


@pytest.mark.parametrize("name", ["c0", "tiny3", "slab_small"])
@pytest.mark.parametrize("precision", [0, 1, 2])
def test_stored_level_values_against_fp64(systems, name, precision):
    """Every smoothed level's operator as the fast path stores it, against the FP64 hierarchy: FP64 exact,
    FP32 within FP32 rounding, BF16 (precision 2, levels >= 1) within BF16 rounding of each value -- its
    per-block power-of-two FP32 scale is exact, so each entry is the BF16 rounding of a_ij."""
    s = systems(name) if name != "slab_small" else synth.reservoir_system(30, 110, 12, seed=21, phases=2,
                                                                         channelised_layers=7)
    G = CprGmres(**dict(BASE, precision=precision, fast_smoother=1, flexible=1)).setup(s.ia, s.ja, s.a,
                                                                                       s.block_size)
    for lev in range(G.num_levels() - 1):
        ia, ja, a, _ = G.level_matrix(lev, 0)
        got = G.level_stored_values(lev)
        kind = G.level_info(lev)["storage"]
        assert kind == (0 if precision == 0 else (2 if precision == 2 and lev >= 1 else 1))
        if kind == 0:
            assert np.array_equal(got, a)
        elif kind == 1:
            assert np.array_equal(got, a.astype(np.float32).astype(np.float64))
        else:
            assert np.all(np.abs(got - a) <= 2.0 ** -8 * np.abs(a)), lev
            # the BF16 rounding of each value: at most 8 significant bits
            m, _ = np.frexp(got[got != 0])
            assert np.all(np.abs(m * 256 - np.round(m * 256)) == 0)
    G.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_two_lane_sliced_ell(precision):
    """The sliced ELL with two lanes per row (sell_lanes 2, without autotuning): every operator that
    takes the sliced ELL uses it, the stored values are the hierarchy's (FP64) or their FP32 rounding,
    and the solve reaches the FP64 true residual in about as many iterations as with one lane per row
    (the pair's shuffle changes the order of the row sums)."""
    s = synth.reservoir_system(30, 110, 12, seed=21, phases=2, channelised_layers=7)
    its = {}
    for lanes in (1, 2):
        G = CprGmres(**dict(BASE, precision=precision, fast_smoother=1, flexible=1, autotune=0,
                            sell_lanes=lanes)).setup(s.ia, s.ja, s.a, s.block_size)
        sell = [l for l in G.setup_report().splitlines() if "layout sell" in l]
        assert sell, G.setup_report()
        assert all(("layout sell/2" in l) == (lanes == 2) for l in sell), sell
        for lev in range(G.num_levels() - 1):
            ia, ja, a, _ = G.level_matrix(lev, 0)
            got = G.level_stored_values(lev)
            assert np.array_equal(got, a if precision == 0 else a.astype(np.float32).astype(np.float64)), lev
        x, it, rel, conv = G.solve(s.b)
        G.close()
        assert conv and true_rel(s, x) <= 1.05e-6, (lanes, it, rel)
        its[lanes] = it
    assert abs(its[2] - its[1]) <= 2, its
