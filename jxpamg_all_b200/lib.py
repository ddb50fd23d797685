"""ctypes binding of libjxcpr_b200.so (the product library).

There is no CPU fallback: if the library is missing or CUDA is unavailable
the calls raise.  The binding mirrors include/jxcpr_b200.h one to one.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libjxcpr_b200.so")

c_int, c_double, c_void_p, c_longlong, c_char_p = (ctypes.c_int, ctypes.c_double, ctypes.c_void_p,
                                                   ctypes.c_longlong, ctypes.c_char_p)

_lib = None


class JxcprError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"jxcpr status {status}: {msg}")
        self.status = status


def _declare(lib):
    f = lib.jxcpr_last_error
    f.restype = c_char_p
    lib.jxcpr_bsr_matvec_dev.argtypes = [c_int, c_int, c_longlong, c_void_p, c_void_p, c_void_p, c_double,
                                         c_void_p, c_double, c_void_p, c_int, c_void_p]
    lib.jxcpr_bsr_matvec_dev_f32.argtypes = lib.jxcpr_bsr_matvec_dev.argtypes
    lib.jxcpr_dot_dev.argtypes = [c_longlong, c_void_p, c_void_p, c_void_p, c_void_p]
    lib.jxcpr_dot_dev_noalloc.argtypes = [c_longlong, c_void_p, c_void_p, c_void_p, c_void_p]
    lib.jxcpr_dense_inverse_dev.argtypes = [c_int, c_void_p, c_void_p, c_void_p]
    _declare_solver(lib)
    _declare_mlp(lib)


def load():
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} not built; run `python -m jxpamg_all_b200.build`")
        _lib = ctypes.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def check(status: int) -> None:
    if status != 0:
        raise JxcprError(status, load().jxcpr_last_error().decode(errors="replace"))


def _declare_solver(lib):
    P = c_void_p
    lib.jxcpr_solver_create.argtypes = [ctypes.POINTER(c_void_p)]
    lib.jxcpr_solver_destroy.argtypes = [P]
    lib.jxcpr_solver_set_int.argtypes = [P, c_char_p, c_int]
    lib.jxcpr_solver_set_stream.argtypes = [P, P]
    lib.jxcpr_launch_count.restype = ctypes.c_ulonglong
    lib.jxcpr_solver_set_real.argtypes = [P, c_char_p, c_double]
    lib.jxcpr_solver_setup.argtypes = [P, c_int, c_int, c_longlong, P, P, P, c_int]
    lib.jxcpr_solver_solve.argtypes = [P, P, P, c_int, P, P]
    lib.jxcpr_solver_get_norms.argtypes = [P, P, c_int]
    lib.jxcpr_solver_stats.argtypes = [P, P]
    lib.jxcpr_solver_setup_report.argtypes = [P, ctypes.c_char_p, c_int]
    lib.jxcpr_solver_num_levels.argtypes = [P]
    lib.jxcpr_solver_level_sizes.argtypes = [P, c_int, c_int, P]
    lib.jxcpr_solver_level_matrix.argtypes = [P, c_int, c_int, P, P, P]
    lib.jxcpr_solver_level_cf.argtypes = [P, c_int, P]
    lib.jxcpr_solver_decoupled_values.argtypes = [P, P]
    lib.jxcpr_solver_cpr_apply.argtypes = [P, P, P, c_int]
    lib.jxcpr_solver_vcycle.argtypes = [P, P, P, c_int]
    lib.jxcpr_solver_stage2_sweep.argtypes = [P, P, P, c_int]
    lib.jxcpr_solver_level_info.argtypes = [P, c_int, P, P, P, P]
    lib.jxcpr_solver_stage2_native.argtypes = [P, c_int]
    lib.jxcpr_solver_level_native.argtypes = [P, c_int, c_int, c_int]
    lib.jxcpr_solver_krylov_native.argtypes = [P, c_int, c_int]
    lib.jxcpr_solver_level_stored_values.argtypes = [P, c_int, P]
    lib.jxcpr_solver_apply_bytes.argtypes = [P, P]
    lib.jxcpr_stage2_chunk_order.argtypes = [c_int, c_void_p, c_void_p, c_int, c_void_p, c_int, c_void_p, c_int]
    lib.jxcpr_solver_bilu_sizes.argtypes = [P, P]
    lib.jxcpr_solver_bilu_factors.argtypes = [P, P, P, P]
    lib.jxcpr_solver_bilu_apply.argtypes = [P, P, P, c_int]
    lib.jxcpr_solver_bilu_levels.argtypes = [P, P, P, P]
    lib.jxcpr_solver_level_features.argtypes = [P, c_int, P]
    lib.jxcpr_solver_learned_status.argtypes = [P, P]
    lib.jxcpr_solver_learned_fallbacks.argtypes = [P]
    lib.jxcpr_pool_stats.argtypes = [P]
    lib.jxcpr_batch_setup.argtypes = [c_int, P, P, P, P, P, P, P, c_int, c_int, P]
    lib.jxcpr_batch_create.argtypes = [ctypes.POINTER(c_void_p), c_int, P]
    lib.jxcpr_batch_destroy.argtypes = [P]
    lib.jxcpr_batch_solve.argtypes = [P, P, P, c_int, P, P, P, P, P]
    lib.jxcpr_batch_last_ms.argtypes = [P, P]
    lib.jxcpr_batch_launch.argtypes = [P, P]


def _declare_mlp(lib):
    P = c_void_p
    lib.jxcpr_mlp_set_weights.argtypes = [P]
    lib.jxcpr_mlp_get_weights.argtypes = [P]
    lib.jxcpr_mlp_forward_host.argtypes = [P, P, P]
    lib.jxcpr_mlp_forward.argtypes = [P, P, c_int, P, P, P]
    lib.jxcpr_mlp_loss_grad.argtypes = [P, P, P, c_int, P, P, P, P]
    lib.jxcpr_mlp_adam.argtypes = [P, P, P, P, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                   c_int, P]
