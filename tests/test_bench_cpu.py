"""Host-side composition of the benchmark's method choices (no GPU).

The measured path of each workload takes the options stated beside it: on C1 the
reference mixed driver's stage-2 weights with the learned settings; on the
three-phase C4 True-IMPES, GMRES(60), the plain CPR weights and no learned
model; the plain FP64 path always keeps the reference CPR's weights and its
host-driven GMRES.
"""
import os
import sys
from types import SimpleNamespace

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_c1_measured_and_plain_options():
    args = SimpleNamespace(config="c1", opt=[])
    m, p = bench.solver_opts(args), bench.plain_opts(args)
    assert (m["stage2_relax_weight"], m["stage2_omega"]) == (1.0, 0.8)
    assert m["precision"] == 1 and m["fast_smoother"] == 2 and m["flexible"] == 1 and m["graph_gmres"] == 1
    assert p["precision"] == 0 and p["fast_smoother"] == 0
    assert "stage2_relax_weight" not in p and p.get("graph_gmres", 0) == 0
    assert m["tol"] == p["tol"] == 1e-6 and m["k_dim"] == p["k_dim"] == 30


def test_c4_measured_and_plain_options():
    args = SimpleNamespace(config="c4", opt=[])
    m, p = bench.solver_opts(args), bench.plain_opts(args)
    for o in (m, p):
        assert o["decouple"] == 5 and o["k_dim"] == 60 and o["max_iter"] == 1000
    assert (m["stage2_relax_weight"], m["stage2_omega"]) == (0.7, 0.9) and m["fast_smoother"] == 2
    assert "stage2_relax_weight" not in p


def test_option_overrides_from_the_command_line():
    args = SimpleNamespace(config="c1", opt=["dep_launch=0", "stage2_omega=0.85"])
    m = bench.solver_opts(args)
    assert m["dep_launch"] == 0 and m["stage2_omega"] == 0.85


def test_measured_path_text_follows_the_options():
    c1 = bench.measured_path_text(bench.solver_opts(SimpleNamespace(config="c1", opt=[])), {"learned_used": True})
    c4 = bench.measured_path_text(bench.solver_opts(SimpleNamespace(config="c4", opt=[])), {"learned_used": False})
    assert "mixed driver's weights 1.0/0.8" in c1 and "(kept)" in c1
    assert "plain CPR's weights 0.7/0.9" in c4 and "rejected by the probe" in c4
    c4d = bench.measured_path_text(bench.solver_opts(SimpleNamespace(config="c4", opt=["fast_smoother=1"])),
                                   {"learned_used": False})
    assert "no learned settings" in c4d


def test_both_arms_print_the_same_config():
    """The reference arm and our arm emit identical `config` objects for a workload, so that a
    comparison of the two lines is like for like."""
    for cfg in ("c1", "c4"):
        args = SimpleNamespace(config=cfg, opt=[])
        assert bench.common_config(cfg, bench.plain_opts(args)) == bench.common_config(cfg, bench.solver_opts(args))
