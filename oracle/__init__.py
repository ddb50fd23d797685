"""ORACLE (test infrastructure only).

ctypes front end to
  * ``liborc.so``      -- the plain-C restatement of the reference CPR-GMRES
                          path (this directory's *.c files), and
  * ``_ref/libjxf_ref64.so`` -- the reference JXFPAMG library compiled from
                          its own sources (FP64) by ``ref.mk``, present when
                          the reference tree was available at build time.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker / baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_LIB = os.path.join(HERE, "liborc.so")
REF_LIB = os.path.join(HERE, "_ref", "libjxf_ref64.so")
REF_TREE = "/root/reference"

_orc = None
_ref = None

c_int, c_double, c_void_p, c_longlong = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_longlong


def _p(a):
    return None if a is None else a.ctypes.data_as(c_void_p)


def build(reference: bool = True, jobs: int = 8) -> None:
    """Compile the restatement; also the reference library when its tree exists."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if reference and os.path.isdir(REF_TREE):
        subprocess.run(["make", "-s", "-f", os.path.join(HERE, "ref.mk"), f"REF={REF_TREE}", f"-j{jobs}"],
                       check=True, cwd=os.path.dirname(HERE))


def orc():
    global _orc
    if _orc is None:
        if not os.path.exists(ORC_LIB):
            build(reference=False)
        _orc = ctypes.CDLL(ORC_LIB)
    return _orc


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError("reference library not built (oracle/_ref/libjxf_ref64.so missing)")
        _ref = ctypes.CDLL(REF_LIB)
        _ref.ref_cpr_create.restype = c_void_p
    return _ref


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ---- restatement ---------------------------------------------------------------
def bsr_matvec(ia, ja, a, bs, x, alpha=1.0, y=None, beta=0.0):
    nb = len(ia) - 1
    ia, ja, a, x = _i32(ia), _i32(ja), _f64(a), _f64(x)
    y = np.zeros(nb * bs) if y is None else _f64(y).copy()
    orc().orc_bsr_matvec(c_int(nb), c_int(bs), _p(ia), _p(ja), _p(a), c_double(alpha), _p(x), c_double(beta),
                         _p(y))
    return y


def bsr_decouple(ia, ja, a, bs, rhs, dtype_code, consistent_rhs=False):
    """Returns (a', rhs') after jxf_BSRMatrixDecouple (1 = ABF, 5 = TIMPES)."""
    nb = len(ia) - 1
    ia, ja = _i32(ia), _i32(ja)
    a2, r2 = _f64(a).copy(), _f64(rhs).copy()
    st = orc().orc_bsr_decouple(c_int(nb), c_int(bs), _p(ia), _p(ja), _p(a2), _p(r2), c_int(dtype_code),
                                c_int(1 if consistent_rhs else 0))
    if st:
        raise ValueError(f"orc_bsr_decouple status {st}")
    return a2, r2


# ---- reference library ------------------------------------------------------------
def ref_bsr_matvec(ia, ja, a, bs, x, alpha=1.0, y=None, beta=0.0):
    nb = len(ia) - 1
    ia, ja, a, x = _i32(ia), _i32(ja), _f64(a), _f64(x)
    y = np.zeros(nb * bs) if y is None else _f64(y).copy()
    ref().ref_bsr_matvec(c_int(nb), c_int(bs), _p(ia), _p(ja), _p(a), c_double(alpha), _p(x), c_double(beta),
                         _p(y))
    return y


def ref_bsr_decouple(ia, ja, a, bs, rhs, dtype_code):
    nb = len(ia) - 1
    ia, ja = _i32(ia), _i32(ja)
    a2, r2 = _f64(a).copy(), _f64(rhs).copy()
    ref().ref_bsr_decouple(c_int(nb), c_int(bs), _p(ia), _p(ja), _p(a2), _p(r2), c_int(dtype_code), c_int(1))
    return a2, r2
