"""ORACLE (test infrastructure only).

ctypes front end to
  * ``liborc.so``      -- the plain-C restatement of the reference CPR-GMRES
                          path (this directory's *.c files), and
  * ``_ref/libjxf_ref64.so`` -- the reference JXFPAMG library compiled from
                          its own sources (FP64) by ``ref.mk``, present when
                          the reference tree was available at build time.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the test oracle / baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_LIB = os.path.join(HERE, "liborc.so")
REF_LIB = os.path.join(HERE, "_ref", "libjxf_ref64.so")
# the reference source tree the test oracle's library is compiled from (build step only)
REF_TREE = os.environ.get("JXF_REFERENCE_TREE", "")

_orc = None
_ref = None

c_int, c_double, c_void_p, c_longlong = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_longlong


def _p(a):
    return None if a is None else a.ctypes.data_as(c_void_p)


def build(reference: bool = True, jobs: int = 8) -> None:
    """Compile the restatement; also the reference library when its tree exists."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    tree = os.environ.get("JXF_REFERENCE_TREE", REF_TREE)
    if reference and tree and os.path.isdir(tree):
        subprocess.run(["make", "-s", "-f", os.path.join(HERE, "ref.mk"), f"REF={tree}", f"-j{jobs}"],
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
def strength(ia, ja, a, theta=0.25, max_row_sum=0.9):
    """Strength pattern (sia, sja) of a CSR operator (par_strength.c rules)."""
    ia, ja, a = _i32(ia), _i32(ja), _f64(a)
    n = len(ia) - 1
    sia = np.zeros(n + 1, np.int32)
    nnz = orc().orc_strength_csr(c_int(n), _p(ia), _p(ja), _p(a), c_double(theta), c_double(max_row_sum),
                                 _p(sia), None)
    sja = np.zeros(max(nnz, 1), np.int32)
    orc().orc_strength_csr(c_int(n), _p(ia), _p(ja), _p(a), c_double(theta), c_double(max_row_sum), _p(sia),
                           _p(sja))
    return sia, sja[:nnz]


def rs_first_pass(sia, sja, range_rows=0):
    """Markers of the Ruge-Stueben first pass on a strength pattern (row ranges when > 0)."""
    sia, sja = _i32(sia), _i32(sja)
    n = len(sia) - 1
    cf = np.zeros(n, np.int32)
    orc().orc_rs_first_pass_csr(c_int(n), _p(sia), _p(sja), c_int(range_rows), _p(cf))
    return cf


def ref_rs_first_pass(sia, sja):
    """The reference's first pass (jxf_PAMGCoarsenRuge, coarsen_type 10) on a strength pattern."""
    sia, sja = _i32(sia), _i32(sja)
    n = len(sia) - 1
    cf = np.zeros(n, np.int32)
    if ref().ref_rs_first_pass(c_int(n), _p(sia), _p(sja if len(sja) else np.zeros(1, np.int32)), _p(cf)) != 0:
        raise RuntimeError("reference first pass failed")
    return cf


def hmis_cf(ia, ja, a, theta=0.25, max_row_sum=0.9, range_rows=0):
    """C/F splitting of a CSR operator: strength, the Ruge-Stueben first pass (on row ranges of
    range_rows rows when > 0) and the PMIS pass; C points 1, F points -1."""
    ia, ja, a = _i32(ia), _i32(ja), _f64(a)
    n = len(ia) - 1
    cf = np.zeros(n, np.int32)
    orc().orc_hmis_ranges(c_int(n), _p(ia), _p(ja), _p(a), c_double(theta), c_double(max_row_sum),
                          c_int(range_rows), _p(cf))
    return cf


def bsr_matvec(ia, ja, a, bs, x, alpha=1.0, y=None, beta=0.0):
    nb = len(ia) - 1
    ia, ja, a, x = _i32(ia), _i32(ja), _f64(a), _f64(x)
    y = np.zeros(nb * bs) if y is None else _f64(y).copy()
    orc().orc_bsr_matvec(c_int(nb), c_int(bs), _p(ia), _p(ja), _p(a), c_double(alpha), _p(x), c_double(beta),
                         _p(y))
    return y


def bsr_decouple(ia, ja, a, bs, rhs, dtype_code, consistent_rhs=False, thermal=False):
    """Returns (a', rhs') after jxf_BSRMatrixDecouple (1 ABF, 2 ANL, 3 SEM, 4 QI, 5 TIMPES,
    6 TIMPES2; thermal applies to 2-4)."""
    nb = len(ia) - 1
    ia, ja = _i32(ia), _i32(ja)
    a2, r2 = _f64(a).copy(), _f64(rhs).copy()
    st = orc().orc_bsr_decouple2(c_int(nb), c_int(bs), _p(ia), _p(ja), _p(a2), _p(r2), c_int(dtype_code),
                                 c_int(1 if thermal else 0), c_int(1 if consistent_rhs else 0))
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


def ref_bsr_decouple(ia, ja, a, bs, rhs, dtype_code, thermal=False):
    nb = len(ia) - 1
    ia, ja = _i32(ia), _i32(ja)
    a2, r2 = _f64(a).copy(), _f64(rhs).copy()
    ref().ref_bsr_decouple2(c_int(nb), c_int(bs), _p(ia), _p(ja), _p(a2), _p(r2), c_int(dtype_code),
                            c_int(1 if thermal else 0), c_int(1))
    return a2, r2


def chunk_colour(ia, ja, chunk):
    """Colour of each block row's chunk in the throughput path's stage-2 order, and the colour count."""
    ia, ja = _i32(ia), _i32(ja)
    nb = len(ia) - 1
    colour = np.zeros(max(nb, 1), np.int32)
    nc = orc().orc_chunk_colour(c_int(nb), _p(ia), _p(ja if len(ja) else np.zeros(1, np.int32)), c_int(chunk),
                                _p(colour))
    return colour[:nb], int(nc)


def hgs_relax_chunked(ia, ja, a, bs, x, b, chunk, w=0.7, omega=0.9):
    """One stage-2 sweep (the reference's weighted block update) in the chunk order."""
    nb = len(ia) - 1
    colour, nc = chunk_colour(ia, ja, chunk)
    x = _f64(x).copy()
    keep = (_i32(ia), _i32(ja), _f64(a))
    orc().orc_hgs_relax_chunked(c_int(nb), c_int(bs), *(_p(v) for v in keep), _p(x), _p(_f64(b)), c_double(w),
                                c_double(omega), c_int(chunk), _p(colour), c_int(nc))
    return x


# ---- AMG / CPR / GMRES handles ----------------------------------------------------
class _CprBase:
    """Common accessors for a CPR handle (restatement or reference)."""

    _prefix = ""

    def _fn(self, name):
        return getattr(self._lib, self._prefix + name)

    def num_levels(self):
        return int(self._fn("cpr_num_levels")(c_void_p(self.h)))

    def level_matrix(self, lev, what):
        """(ia, ja, a) of A_l (what=0) or P_l (what=1), or None."""
        sizes = np.zeros(3, np.int32)
        st = self._fn("cpr_level_sizes")(c_void_p(self.h), c_int(lev), c_int(what), _p(sizes))
        if st < 0:
            return None
        n, m, nnz = (int(v) for v in sizes)
        ia = np.zeros(n + 1, np.int32)
        ja = np.zeros(max(nnz, 1), np.int32)
        a = np.zeros(max(nnz, 1))
        self._fn("cpr_level_matrix")(c_void_p(self.h), c_int(lev), c_int(what), _p(ia), _p(ja), _p(a))
        return ia, ja[:nnz], a[:nnz], m

    def level_cf(self, lev, n):
        cf = np.zeros(n, np.int32)
        st = self._fn("cpr_level_cf")(c_void_p(self.h), c_int(lev), _p(cf))
        return None if st < 0 else cf


class OracleCPR(_CprBase):
    """CPR setup of the restatement (AMG hierarchy built at construction)."""

    _prefix = "orc_"

    def __init__(self, ia, ja, a, bs, stage2_maxit=3, stage2_type=2, stage2_chunk=0):
        self._lib = orc()
        self._lib.orc_cpr_create.restype = c_void_p
        self.nb, self.bs = len(ia) - 1, bs
        self._keep = (_i32(ia), _i32(ja), _f64(a))
        self.h = self._lib.orc_cpr_create(c_int(self.nb), c_int(bs), *(_p(v) for v in self._keep),
                                          c_int(stage2_maxit))
        self._lib.orc_cpr_set_stage2_type(c_void_p(self.h), c_int(stage2_type))
        if stage2_chunk:
            self._lib.orc_cpr_set_stage2_chunk_h(c_void_p(self.h), c_int(stage2_chunk))

    def apply(self, r):
        z = np.zeros(self.nb * self.bs)
        self._lib.orc_cpr_apply_h(c_void_p(self.h), _p(_f64(r)), _p(z))
        return z

    def vcycle(self, rp, xp=None):
        xp = np.zeros(self.nb) if xp is None else _f64(xp).copy()
        self._lib.orc_cpr_amg_vcycle(c_void_p(self.h), _p(_f64(rp)), _p(xp))
        return xp

    def __del__(self):
        try:
            self._lib.orc_cpr_destroy(c_void_p(self.h))
        except Exception:
            pass


class RefCPR(_CprBase):
    """CPR setup of the reference library (JXF_CPRCreate/SetParameter/Setup)."""

    _prefix = "ref_"

    def __init__(self, ia, ja, a, bs, stage2_maxit=3, stage2_type=2):
        self._lib = ref()
        self.nb, self.bs = len(ia) - 1, bs
        self._keep = (_i32(ia), _i32(ja), _f64(a))
        self.h = self._lib.ref_cpr_create(c_int(self.nb), c_int(bs), *(_p(v) for v in self._keep), c_int(1),
                                          c_int(stage2_maxit), c_int(stage2_type), c_int(1))
        if not self.h:
            raise RuntimeError("reference CPR setup failed")

    def apply(self, r):
        z = np.zeros(self.nb * self.bs)
        self._lib.ref_cpr_apply(c_void_p(self.h), _p(_f64(r)), _p(z), c_int(1))
        return z

    def vcycle(self, rp, xp=None):
        xp = np.zeros(self.nb) if xp is None else _f64(xp).copy()
        self._lib.ref_cpr_amg_solve(c_void_p(self.h), _p(_f64(rp)), _p(xp), c_int(1))
        return xp


def gmres(ia, ja, a, bs, b, x0=None, k_dim=30, tol=1e-6, max_iter=200, cpr=None):
    """Restated GMRES; returns dict(x, iters, rel, converged, norms)."""
    nb = len(ia) - 1
    n = nb * bs
    x = np.zeros(n) if x0 is None else _f64(x0).copy()
    rel = np.zeros(1)
    conv = np.zeros(1, np.int32)
    norms = np.zeros(max_iter + 1)
    keep = (_i32(ia), _i32(ja), _f64(a), _f64(b))
    it = orc().orc_gmres_solve(c_int(nb), c_int(bs), *(_p(v) for v in keep), _p(x), c_int(k_dim),
                               c_double(tol), c_int(max_iter), c_void_p(cpr.h if cpr else 0), _p(rel), _p(conv),
                               _p(norms))
    return dict(x=x, iters=int(it), rel=float(rel[0]), converged=bool(conv[0]), norms=norms[:it + 1])


def ref_gmres(ia, ja, a, bs, b, x0=None, k_dim=30, tol=1e-6, max_iter=200, decouple=0, precond=1,
              stage2_maxit=3, stage2_type=2):
    """The reference driver sequence (decouple -> CPR setup -> GMRES solve)."""
    nb = len(ia) - 1
    n = nb * bs
    x = np.zeros(n) if x0 is None else _f64(x0).copy()
    info = np.zeros(2, np.int32)
    rel = np.zeros(2)
    norms = np.zeros(max_iter + 1)
    times = np.zeros(5)
    keep = (_i32(ia), _i32(ja), _f64(a), _f64(b))
    ref().ref_cpr_gmres_solve(c_int(nb), c_int(bs), *(_p(v) for v in keep), _p(x), c_int(decouple),
                              c_int(precond), c_int(k_dim), c_double(tol), c_int(max_iter), c_int(stage2_maxit),
                              c_int(stage2_type), _p(info), _p(rel), _p(norms), _p(times), c_int(1))
    it = int(info[0])
    return dict(x=x, iters=it, rel=float(rel[0]), true_rel=float(rel[1]), converged=bool(info[1]),
                norms=norms[:it + 1], times=times)


def hgs_relax(ia, ja, a, bs, x, b, w=0.7, omega=0.9, direction=1, sweeps=1):
    nb = len(ia) - 1
    x = _f64(x).copy()
    keep = (_i32(ia), _i32(ja), _f64(a))
    for _ in range(sweeps):
        orc().orc_hgs_relax(c_int(nb), c_int(bs), *(_p(v) for v in keep), _p(x), _p(_f64(b)), c_double(w),
                            c_double(omega), c_int(direction))
    return x


def ref_hgs_relax(ia, ja, a, bs, x, b, w=0.7, omega=0.9, direction=1, sweeps=1):
    nb = len(ia) - 1
    x = _f64(x).copy()
    keep = (_i32(ia), _i32(ja), _f64(a))
    ref().ref_hgs_relax(c_int(nb), c_int(bs), *(_p(v) for v in keep), _p(x), _p(_f64(b)), c_double(w),
                        c_double(omega), c_int(direction), c_int(sweeps))
    return x


def hsgs_relax(ia, ja, a, bs, x, b, work, w=0.7, omega=0.9, sweeps=1):
    """jxf_ParBSRHSGSRelax restated; returns (x, work) (work = the Vtemp vector, in/out)."""
    nb = len(ia) - 1
    x, work = _f64(x).copy(), _f64(work).copy()
    keep = (_i32(ia), _i32(ja), _f64(a))
    for _ in range(sweeps):
        orc().orc_hsgs_relax(c_int(nb), c_int(bs), *(_p(v) for v in keep), _p(x), _p(_f64(b)), _p(work),
                             c_double(w), c_double(omega))
    return x, work


def ref_hsgs_relax(ia, ja, a, bs, x, b, work, w=0.7, omega=0.9, sweeps=1):
    nb = len(ia) - 1
    x, work = _f64(x).copy(), _f64(work).copy()
    keep = (_i32(ia), _i32(ja), _f64(a))
    ref().ref_hsgs_relax(c_int(nb), c_int(bs), *(_p(v) for v in keep), _p(x), _p(_f64(b)), _p(work),
                         c_double(w), c_double(omega), c_int(sweeps))
    return x, work


# ---- block ILU(0) (orc_bilu.c restatement; ref_bilu = the reference library) ---------
def bilu_pattern(ia, ja):
    """Strictly lower / upper block patterns of A in A's entry order: (lia, lja, uia, uja)."""
    nb = len(ia) - 1
    ia, ja = _i32(ia), _i32(ja)
    lia, uia = np.zeros(nb + 1, np.int32), np.zeros(nb + 1, np.int32)
    lja, uja = np.zeros(max(len(ja), 1), np.int32), np.zeros(max(len(ja), 1), np.int32)
    orc().orc_bilu_pattern(c_int(nb), _p(ia), _p(ja), _p(lia), _p(lja), _p(uia), _p(uja))
    return lia, lja[:lia[-1]].copy(), uia, uja[:uia[-1]].copy()


def bilu_setup(ia, ja, a, bs, sweeps=3):
    """Factors of jxf_ILUSetupFGPBILU_v3: dict(lia, lja, la, uia, uja, ua, dinv)."""
    nb = len(ia) - 1
    lia, lja, uia, uja = bilu_pattern(ia, ja)
    bn = bs * bs
    la = np.zeros(max(len(lja), 1) * bn)
    ua = np.zeros(max(len(uja), 1) * bn)
    dinv = np.zeros(nb * bn)
    orc().orc_bilu_setup(c_int(nb), c_int(bs), _p(_i32(ia)), _p(_i32(ja)), _p(_f64(a)), c_int(sweeps), _p(lia),
                         _p(lja), _p(la), _p(uia), _p(uja), _p(ua), _p(dinv))
    return dict(lia=lia, lja=lja, la=la[:len(lja) * bn], uia=uia, uja=uja, ua=ua[:len(uja) * bn], dinv=dinv)


def bilu_solve(ia, ja, a, bs, F, f, ir=5, lower=5, upper=5, u0=None):
    """u = BILU(f) with tri-solve 14 (u0 = 0 unless given)."""
    nb = len(ia) - 1
    u = np.zeros(nb * bs) if u0 is None else _f64(u0).copy()
    orc().orc_bilu_solve(c_int(nb), c_int(bs), _p(_i32(ia)), _p(_i32(ja)), _p(_f64(a)), _p(F["lia"]),
                         _p(F["lja"]), _p(F["la"]), _p(F["uia"]), _p(F["uja"]), _p(F["ua"]), _p(F["dinv"]),
                         c_int(ir), c_int(lower), c_int(upper), _p(_f64(f)), _p(u))
    return u


def bilu_levels(ia, ja):
    """Levels of the lower and upper block-triangular DAGs: (lev_l, lev_u, number of lower levels,
    number of upper levels)."""
    nb = len(ia) - 1
    lia, lja, uia, uja = bilu_pattern(ia, ja)
    lev_l, lev_u = np.zeros(max(nb, 1), np.int32), np.zeros(max(nb, 1), np.int32)
    nup = np.zeros(1, np.int32)
    nl = orc().orc_bilu_levels(c_int(nb), _p(lia), _p(lja if len(lja) else np.zeros(1, np.int32)), _p(uia),
                               _p(uja if len(uja) else np.zeros(1, np.int32)), _p(lev_l), _p(lev_u), _p(nup))
    return lev_l[:nb], lev_u[:nb], int(nl), int(nup[0])


def bilu_setup_exact(ia, ja, a, bs):
    """Exact block ILU(0) factors (the fixed point of jxf_ILUSetupFGPBILU_v3's sweeps), as bilu_setup."""
    nb = len(ia) - 1
    lia, lja, uia, uja = bilu_pattern(ia, ja)
    bn = bs * bs
    la = np.zeros(max(len(lja), 1) * bn)
    ua = np.zeros(max(len(uja), 1) * bn)
    dinv = np.zeros(nb * bn)
    orc().orc_bilu_setup_exact(c_int(nb), c_int(bs), _p(_i32(ia)), _p(_i32(ja)), _p(_f64(a)), _p(lia),
                               _p(lja if len(lja) else np.zeros(1, np.int32)), _p(la), _p(uia),
                               _p(uja if len(uja) else np.zeros(1, np.int32)), _p(ua), _p(dinv))
    return dict(lia=lia, lja=lja, la=la[:len(lja) * bn], uia=uia, uja=uja, ua=ua[:len(uja) * bn], dinv=dinv)


def bilu_solve_exact(ia, ja, a, bs, F, f, ir=5, u0=None):
    """u += BILU^-1 (f - A u) with substitution in level order, `ir` refinement loops."""
    nb = len(ia) - 1
    u = np.zeros(nb * bs) if u0 is None else _f64(u0).copy()
    z = np.zeros(1, np.int32)
    orc().orc_bilu_solve_exact(c_int(nb), c_int(bs), _p(_i32(ia)), _p(_i32(ja)), _p(_f64(a)), _p(F["lia"]),
                               _p(F["lja"] if len(F["lja"]) else z), _p(F["la"] if len(F["la"]) else np.zeros(1)),
                               _p(F["uia"]), _p(F["uja"] if len(F["uja"]) else z),
                               _p(F["ua"] if len(F["ua"]) else np.zeros(1)), _p(F["dinv"]), c_int(ir), _p(_f64(f)),
                               _p(u))
    return u


def ref_bilu(ia, ja, a, bs, f, sweeps=3, ir=5, lower=5, upper=5):
    """The reference's jxf_BILUSetup + jxf_BILUSolve: (u, la, ua, dinv)."""
    nb = len(ia) - 1
    lia, lja, uia, uja = bilu_pattern(ia, ja)
    bn = bs * bs
    la = np.zeros(max(len(lja), 1) * bn)
    ua = np.zeros(max(len(uja), 1) * bn)
    dinv = np.zeros(nb * bn)
    u = np.zeros(nb * bs)
    st = ref().ref_bilu(c_int(nb), c_int(bs), _p(_i32(ia)), _p(_i32(ja)), _p(_f64(a)), c_int(sweeps), c_int(ir),
                        c_int(lower), c_int(upper), _p(_f64(f)), _p(u), _p(la), _p(ua), _p(dinv), c_int(1))
    if st:
        raise RuntimeError(f"ref_bilu returned {st}")
    return u, la[:len(lja) * bn], ua[:len(uja) * bn], dinv


def cpr_bilu_apply(cpr, ia, ja, a, bs, F, r, ir=5, lower=5, upper=5):
    """Stage-2 BILU composition: z = CPR(r) without stage-2 sweeps, r' = r - A z, z += BILU(r')."""
    z = cpr.apply(r)
    rr = bsr_matvec(ia, ja, a, bs, z, alpha=-1.0, y=_f64(r).copy(), beta=1.0)
    return z + 1.0 * bilu_solve(ia, ja, a, bs, F, rr, ir, lower, upper)
