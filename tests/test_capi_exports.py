"""The C-ABI library loads on a CPU-only machine and exports every function
that include/*.h declares (no compute call is made here)."""
import ctypes
import glob
import os
import re

from jxpamg_all_b200 import lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = "\n".join(l for l in text.splitlines() if not l.lstrip().startswith("#"))
        for m in re.finditer(r"JXCPR_API\s+[^;(]*?\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_something():
    assert len(declared_functions()) >= 5


def test_library_exports_every_declared_symbol():
    so = lib.load()
    missing = [n for n in declared_functions() if not hasattr(so, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_version_and_error_without_gpu():
    so = lib.load()
    assert so.jxcpr_version() >= 10000
    assert isinstance(so.jxcpr_last_error(), bytes)


INT_KEYS = ["k_dim", "max_iter", "min_iter", "is_check_restarted", "print_level", "logging", "pressure_index",
            "stage1_maxit", "stage2_maxit", "stage1_solver_type", "stage2_solver_type", "decouple", "thermal",
            "consistent_rhs", "smoother_order", "coarse_exact", "max_colors", "rs_range_rows", "rs_range_rows_coarse", "dep_launch",
            "use_tma_spmv", "precision", "bf16_level", "fast_smoother", "stage2_lanes", "stage2_chunk", "tail_rows", "tail_ctas", "sell_lanes", "learned_fallback",
            "record_features", "flexible", "autotune", "graphs", "orthog", "graph_gmres", "krylov_fp32", "selective_reorth", "bilu_sweeps",
            "bilu_ir_iters", "bilu_lower_iters", "bilu_upper_iters", "bilu_exact"]
REAL_KEYS = ["tol", "a_tol", "threshold", "convfac_threshold", "stage2_relax_weight", "stage2_omega",
             "strong_threshold", "strong_threshold_coarse", "cheb_lower", "cheb_upper", "jacobi_mean_row"]


VALID_INT = {"stage2_chunk": 8}


def test_option_keys_accepted_and_documented():
    """Every option key is taken by jxcpr_solver_set_int / _set_real (host-side only: no device
    work before setup), unknown keys return 4 as JXF_CPRSetParameter does, and each key is
    described in the public header."""
    so = lib.load()
    so.jxcpr_solver_set_int.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
    so.jxcpr_solver_set_real.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_double]
    so.jxcpr_solver_destroy.argtypes = [ctypes.c_void_p]
    h = ctypes.c_void_p()
    assert so.jxcpr_solver_create(ctypes.byref(h)) == 0
    header = open(os.path.join(ROOT, "include", "jxcpr_b200.h")).read()
    try:
        for k in INT_KEYS:
            assert so.jxcpr_solver_set_int(h, k.encode(), VALID_INT.get(k, 1)) == 0, k
            assert re.search(r"\b%s\b" % k, header), f"{k} not described in jxcpr_b200.h"
        for k in REAL_KEYS:
            assert so.jxcpr_solver_set_real(h, k.encode(), 0.5) == 0, k
            assert re.search(r"\b%s\b" % k, header), f"{k} not described in jxcpr_b200.h"
        assert so.jxcpr_solver_set_int(h, b"stage2_chunk", 5) == 4  # chunks must tile the 32-row slices
        assert so.jxcpr_solver_set_int(h, b"no_such_key", 1) == 4
        assert so.jxcpr_solver_set_real(h, b"no_such_key", 1.0) == 4
    finally:
        so.jxcpr_solver_destroy(h)
