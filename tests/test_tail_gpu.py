"""The small coarse levels of the fast V-cycle fused into one cooperative kernel (tail_rows): the
same passes in the same order with the same per-row arithmetic as one launch per pass, so the
V-cycle and the whole solve are bit-identical to the unfused ones, for every smoother kind and
storage precision of the fast path."""
import numpy as np
import pytest

from jxpamg_all_b200.solver import CprGmres

pytestmark = pytest.mark.gpu

BASE = dict(decouple=1, smoother_order=1, coarse_exact=0)
VARIANTS = {
    "fp64-gs-jacobi": dict(precision=0, fast_smoother=0),
    "fp32-chebyshev": dict(precision=1, fast_smoother=1, flexible=1),
    "fp32-cheb-everywhere": dict(precision=1, fast_smoother=3, flexible=1),
    "bf16-levels": dict(precision=2, bf16_level=1, fast_smoother=1, flexible=1),
    "learned": dict(precision=1, fast_smoother=2, flexible=1),
    "graph-gmres-fp32-basis": dict(precision=1, fast_smoother=2, flexible=1, graph_gmres=1, krylov_fp32=1),
}


def make(s, tail_rows, **opt):
    return CprGmres(**dict(BASE, tail_rows=tail_rows, **opt)).setup(s.ia, s.ja, s.a, s.block_size)


@pytest.mark.parametrize("name", ["small", "c0", "tiny3"])
@pytest.mark.parametrize("variant", sorted(VARIANTS))
def test_fused_tail_is_bit_identical(systems, name, variant):
    s = systems(name)
    opt = VARIANTS[variant]
    rp = np.random.default_rng(11).standard_normal(s.num_block_rows)
    out = {}
    for tr in (0, 1 << 30, 2000):  # off; every level from level 1; only the levels below 2,000 rows
        G = make(s, tr, **opt)
        v = G.vcycle(rp)
        x, it, rel, conv = G.solve(s.b)
        out[tr] = (v, x, it, conv)
        G.close()
    for tr in (1 << 30, 2000):
        assert np.array_equal(out[tr][0], out[0][0]), (variant, tr, "V-cycle")
        assert out[tr][2] == out[0][2] and out[tr][3] == out[0][3]
        assert np.array_equal(out[tr][1], out[0][1]), (variant, tr, "solution")


def test_fused_tail_on_c1_levels(systems):
    """The config-1 hierarchy with its small levels fused: the measured path's V-cycle unchanged."""
    from jxpamg_all_b200 import synth

    import bench

    s = synth.config_system("c1")
    opts = dict(bench.SOLVER_OPTS)
    rp = np.random.default_rng(3).standard_normal(s.num_block_rows)
    vs = []
    for tr in (0, 40000):
        G = CprGmres(**dict(opts, tail_rows=tr)).setup(s.ia, s.ja, s.a, s.block_size)
        vs.append(G.vcycle(rp))
        G.close()
    assert np.array_equal(vs[0], vs[1])
