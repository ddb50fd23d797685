"""Device-side GMRES (graph_gmres) and batched solves in one graph launch.

graph_gmres runs the whole restarted flexible GMRES on the device (conditional
graph nodes, two-pass classical Gram-Schmidt, true-residual restarts), so it
is checked through what the method guarantees: the TRUE FP64 residual of the
decoupled system (recomputed on the CPU with the oracle) is below the
tolerance, the iteration count stays within 10 % of the host GMRES with the
same preconditioner, and replays are deterministic.  A batch records the same
kernels per system into one graph, so every system's solution must be
bit-identical to its own single-system graph solve.
"""
import numpy as np
import pytest

import oracle
from jxpamg_all_b200 import synth
from jxpamg_all_b200.lib import JxcprError
from jxpamg_all_b200.solver import CprGmres, CprGmresBatch, STATUS_CONV, setup_many

pytestmark = pytest.mark.gpu

MIXED = dict(decouple=1, max_iter=400, smoother_order=1, coarse_exact=0, precision=1, fast_smoother=1, flexible=1)


def true_rel(s, x, decouple=1):
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, decouple)
    r = b - synth.bsr_matvec_np(s.ia, s.ja, a, s.block_size, x)
    return np.linalg.norm(r) / np.linalg.norm(b)


def make(s, **opt):
    return CprGmres(**dict(MIXED, **opt)).setup(s.ia, s.ja, s.a, s.block_size)


def slab_small():
    return synth.reservoir_system(30, 110, 12, seed=21, phases=2, channelised_layers=7)


VARIANTS = [
    dict(),
    dict(precision=0, fast_smoother=0, flexible=0),
    dict(precision=1, fast_smoother=2),
    dict(precision=2, fast_smoother=1),
    dict(k_dim=8),
    dict(krylov_fp32=1),
    dict(precision=0, fast_smoother=0, flexible=0, krylov_fp32=1),
    dict(k_dim=8, krylov_fp32=1),
    dict(selective_reorth=1),
    dict(krylov_fp32=1, selective_reorth=1),
]


@pytest.mark.parametrize("name", ["small", "c0", "tiny3", "slab_small"])
@pytest.mark.parametrize("opt", VARIANTS, ids=lambda o: "-".join(f"{k}{v}" for k, v in o.items()) or "mixed")
def test_graph_gmres_reaches_true_residual(systems, name, opt):
    s = systems(name) if name != "slab_small" else slab_small()
    G = make(s, **opt)
    x_h, it_h, _, conv_h = G.solve(s.b)
    G.set(graph_gmres=1)
    x, it, rel, conv = G.solve(s.b)
    assert conv_h and conv, (it_h, it, rel)
    assert rel <= 1e-6
    assert true_rel(s, x) <= 1.05e-6
    assert abs(it - it_h) <= max(2, int(0.1 * it_h)), (it, it_h)
    assert np.linalg.norm(x - x_h) <= 1e-3 * np.linalg.norm(x_h)
    G.close()


def test_graph_gmres_norm_history(systems):
    s = systems("c0")
    G = make(s, graph_gmres=1, k_dim=10)
    x, it, rel, conv = G.solve(s.b)
    h = G.norms()
    assert conv and len(h) == it + 1
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    assert h[0] == pytest.approx(np.linalg.norm(b), rel=1e-12)  # x0 = 0
    assert h[-1] <= 1e-6 * np.linalg.norm(b) * 1.0000001
    # within a cycle the GMRES estimate never grows
    for c in range(0, it, 10):
        seg = h[c + 1:min(c + 11, it + 1)]
        assert np.all(np.diff(seg) <= 1e-12 * h[0])
    G.close()


def test_graph_gmres_replay_is_deterministic(systems):
    s = systems("small")
    G = make(s, graph_gmres=1)
    x1, it1, rel1, _ = G.solve(s.b)
    x2, it2, rel2, _ = G.solve(s.b)
    assert it1 == it2 and rel1 == rel2 and np.array_equal(x1, x2)
    G.close()


def test_graph_gmres_rebuilds_on_option_change(systems):
    s = systems("c0")
    G = make(s, graph_gmres=1)
    _, it6, rel6, _ = G.solve(s.b)
    G.set(tol=1e-9)
    _, it9, rel9, conv = G.solve(s.b)
    assert conv and rel9 <= 1e-9 and it9 > it6
    G.close()


def test_graph_gmres_max_iter_and_zero_rhs(systems):
    s = systems("c0")
    G = make(s, graph_gmres=1, max_iter=3)
    x, it, rel, conv = G.solve(s.b)
    assert not conv and it == 3 and rel > 1e-6
    G.set(max_iter=400)
    x, it, rel, conv = G.solve(np.zeros_like(s.b))
    assert conv and it == 0 and not np.any(x)
    # a non-zero initial guess is honoured
    x_ref, it_ref, _, _ = G.solve(s.b)
    x, it, rel, conv = G.solve(s.b, x0=x_ref)
    assert conv and it == 0
    G.close()


def test_graph_gmres_needs_fast_path(systems):
    s = systems("tiny")
    G = CprGmres(decouple=1, graph_gmres=1).setup(s.ia, s.ja, s.a, s.block_size)
    with pytest.raises(JxcprError) as e:
        G.solve(s.b)
    assert e.value.status == 4
    G.close()


def batch_set():
    return [synth.config_system("small"), synth.config_system("c0"), synth.config_system("tiny3"),
            synth.reservoir_system(16, 16, 8, 5), slab_small(), synth.reservoir_system(9, 7, 5, 6)]


def test_batch_matches_single_graph_solves():
    systems = batch_set()
    solvers = [make(s, graph_gmres=1) for s in systems]
    single = [G.solve(s.b) for G, s in zip(solvers, systems)]
    B = CprGmresBatch(solvers)
    out = B.solve([s.b for s in systems])
    for k, (x, it, rel, conv) in enumerate(single):
        assert out["iterations"][k] == it
        assert out["rel_residual"][k] == rel
        assert out["status"][k] == (0 if conv else STATUS_CONV)
        assert np.array_equal(out["x"][k], x), k
        assert true_rel(systems[k], out["x"][k]) <= 1.05e-6
    assert np.all(out["latency_ms"] > 0) and np.all(out["finish_ms"] >= out["latency_ms"] * 0.999)
    assert B.last_ms() > 0
    # a second launch gives the same answers
    out2 = B.solve([s.b for s in systems])
    for k in range(len(systems)):
        assert np.array_equal(out2["x"][k], out["x"][k])
    B.close()
    for G in solvers:
        G.close()


def test_batch_device_arrays():
    import torch

    systems = batch_set()[:3]
    solvers = [make(s) for s in systems]
    B = CprGmresBatch(solvers)
    ref = B.solve([s.b for s in systems])
    bd = [torch.tensor(s.b, device="cuda") for s in systems]
    xd = [torch.zeros(s.n, dtype=torch.float64, device="cuda") for s in systems]
    torch.cuda.synchronize()
    out = B.solve([t.data_ptr() for t in bd], [t.data_ptr() for t in xd], device=True)
    for k in range(len(systems)):
        assert np.array_equal(xd[k].cpu().numpy(), ref["x"][k])
        assert out["iterations"][k] == ref["iterations"][k]
    B.close()


def test_batch_workload_sample_converges():
    systems = synth.batch_systems(count=8, grid_max=(28, 30, 14))
    solvers = [make(s, precision=1, fast_smoother=2) for s in systems]
    B = CprGmresBatch(solvers)
    out = B.solve([s.b for s in systems])
    assert np.all(out["status"] == 0)
    for k, s in enumerate(systems):
        assert true_rel(s, out["x"][k]) <= 1.05e-6
    B.close()


def test_batch_rejects_unset_solver(systems):
    s = systems("tiny")
    G = make(s)
    H = CprGmres(**MIXED)
    with pytest.raises(JxcprError) as e:
        CprGmresBatch([G, H])
    assert e.value.status == 4
    G.close()
    H.close()


def test_parallel_setup_matches_sequential():
    """Setups on host threads (one stream per solver) build the same hierarchies: with the layout
    timing off, every solve is bit-identical to the one after a sequential setup."""
    systems = synth.batch_systems(count=10, grid_max=(30, 40, 16))
    opt = dict(MIXED, autotune=0)
    seq = [make(s, **opt) for s in systems]
    par = setup_many([CprGmres(**opt) for _ in systems], systems, threads=6)
    for s, A, B in zip(systems, seq, par):
        xa, ia, ra, ca = A.solve(s.b)
        xb, ib, rb, cb = B.solve(s.b)
        assert ca and cb and ia == ib and np.array_equal(xa, xb)
    for G in seq + par:
        G.close()


def test_parallel_setup_shared_tuning_batch():
    systems = synth.batch_systems(count=12, grid_max=(34, 40, 16))
    solvers = setup_many([CprGmres(**dict(MIXED, autotune=2)) for _ in systems], systems, threads=0)
    B = CprGmresBatch(solvers)
    out = B.solve([s.b for s in systems])
    assert np.all(out["status"] == 0)
    for k, s in enumerate(systems):
        assert true_rel(s, out["x"][k]) <= 1.05e-6
    B.close()
    for G in solvers:
        G.close()


def test_parallel_setup_reports_failure():
    systems = [synth.config_system("tiny"), synth.config_system("small")]
    bad = synth.config_system("tiny")
    bad.block_size = 4  # rejected by the argument check before any device work
    solvers = [CprGmres(**MIXED) for _ in range(3)]
    with pytest.raises(JxcprError) as e:
        setup_many(solvers, systems + [bad], threads=3)
    assert e.value.status == 4 and "system 2" in str(e.value)
    for G in solvers:
        G.close()


def test_krylov_native_after_a_solve(systems):
    """The orthogonalisation kernels queued outside the graph (the profiling / roofline entry point)
    need a device-GMRES solve first, run on the basis it left, and the next solve starts afresh."""
    from jxpamg_all_b200 import lib

    s = systems("c0")
    G = make(s, graph_gmres=1, krylov_fp32=1, k_dim=10)
    so = lib.load()
    assert so.jxcpr_solver_krylov_native(G.h, 3, 1) == 4  # no device-GMRES solve yet
    x0, it0, rel0, conv0 = G.solve(s.b)
    assert so.jxcpr_solver_krylov_native(G.h, 11, 1) == 4  # m > k_dim
    lib.check(so.jxcpr_solver_krylov_native(G.h, 5, 3))
    x1, it1, rel1, conv1 = G.solve(s.b)
    assert conv0 and conv1 and it0 == it1
    assert np.array_equal(x0, x1)
    G.close()

