"""Python front end of the device CPR-GMRES solver object (libjxcpr_b200.so).

Mirrors the reference's setup/solve sequence (decouple -> CPR setup -> GMRES
solve, src/test_bsr_cprgmres.c:123-429) with its option names; host numpy
arrays or device pointers (ints) are accepted.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import lib as _lib

STATUS_CONV = 256


def _ptr(a):
    if isinstance(a, int):
        return ctypes.c_void_p(a)
    return a.ctypes.data_as(ctypes.c_void_p)


class CprGmres:
    """CPR-GMRES solver on the GPU.

    Integer options: k_dim, max_iter, min_iter, is_check_restarted,
    pressure_index, stage1_maxit, stage2_maxit, stage1_solver_type,
    stage2_solver_type, decouple, consistent_rhs, smoother_order, coarse_exact,
    use_tma_spmv, precision, bf16_level, fast_smoother, stage2_lanes, stage2_chunk, tail_rows, tail_ctas, sell_lanes,
    learned_fallback, record_features, flexible, graph_gmres, krylov_fp32,
    selective_reorth.  Real options: tol, a_tol, threshold,
    convfac_threshold, stage2_relax_weight, stage2_omega, strong_threshold,
    cheb_lower, cheb_upper.

    smoother_order 0 is the exact-order path (preconditioner bit-identical to
    the reference); 1 the throughput path, whose precision (0 FP64, 1 FP32,
    2 FP32 + BF16 coarse levels) and fast_smoother (0 multicolour GS /
    l1-Jacobi, 1 Chebyshev-3, 2 learned) select the mixed and learned forms.
    graph_gmres 1 runs the whole GMRES solve on the device as one CUDA graph
    (fast path only); krylov_fp32 1 stores its basis in FP32 and
    selective_reorth 1 takes the second Gram-Schmidt pass only where the first
    cancelled more than half of the new vector's norm.
    """

    def __init__(self, **options):
        self._so = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(self._so.jxcpr_solver_create(ctypes.byref(h)))
        self.h = h
        self.nb = self.bs = 0
        self.set(**options)

    def set_stream(self, stream_handle: int):
        """Run on an existing CUDA stream (e.g. torch.cuda.current_stream().cuda_stream)."""
        _lib.check(self._so.jxcpr_solver_set_stream(self.h, ctypes.c_void_p(stream_handle)))
        return self

    def set(self, **options):
        for k, v in options.items():
            if isinstance(v, float):
                st = self._so.jxcpr_solver_set_real(self.h, k.encode(), float(v))
            else:
                st = self._so.jxcpr_solver_set_int(self.h, k.encode(), int(v))
            _lib.check(st)
        return self

    def setup(self, ia, ja, a, bs, nb=None, nnzb=None, device=False):
        if device:
            self.nb, self.bs = int(nb), int(bs)
            _lib.check(self._so.jxcpr_solver_setup(self.h, self.nb, self.bs, int(nnzb), _ptr(ia), _ptr(ja),
                                                   _ptr(a), 1))
        else:
            self._keep = (np.ascontiguousarray(ia, np.int32), np.ascontiguousarray(ja, np.int32),
                          np.ascontiguousarray(a, np.float64))
            self.nb, self.bs = len(ia) - 1, int(bs)
            _lib.check(self._so.jxcpr_solver_setup(self.h, self.nb, self.bs, len(ja), *(_ptr(v) for v in self._keep),
                                                   0))
        return self

    def solve(self, b, x0=None, device=False):
        """Returns (x, iterations, relative residual, converged)."""
        it = np.zeros(1, np.int32)
        rel = np.zeros(1)
        if device:
            st = self._so.jxcpr_solver_solve(self.h, _ptr(b), _ptr(x0), 1, _ptr(it), _ptr(rel))
            x = x0
        else:
            x = np.zeros(self.nb * self.bs) if x0 is None else np.array(x0, dtype=np.float64)
            bb = np.ascontiguousarray(b, np.float64)
            st = self._so.jxcpr_solver_solve(self.h, _ptr(bb), _ptr(x), 0, _ptr(it), _ptr(rel))
        if st not in (0, STATUS_CONV):
            _lib.check(st)
        return x, int(it[0]), float(rel[0]), st == 0

    def norms(self):
        buf = np.zeros(100000)
        n = self._so.jxcpr_solver_get_norms(self.h, _ptr(buf), len(buf))
        return buf[:n].copy()

    def stats(self):
        s = np.zeros(4)
        _lib.check(self._so.jxcpr_solver_stats(self.h, _ptr(s)))
        return dict(setup_ms=s[0], solve_ms=s[1], cpr_stage1_setup_s=s[2], levels=int(s[3]))

    def setup_report(self):
        buf = ctypes.create_string_buffer(8192)
        self._so.jxcpr_solver_setup_report(self.h, buf, len(buf))
        return buf.value.decode()

    # ---- inspection -----------------------------------------------------------
    def num_levels(self):
        return int(self._so.jxcpr_solver_num_levels(self.h))

    def level_sizes(self, lev, what=0):
        """(rows, cols, nnz) of level lev's operator (what 0), P (1) or R (2)."""
        sz = np.zeros(3, np.int32)
        if self._so.jxcpr_solver_level_sizes(self.h, lev, what, _ptr(sz)) < 0:
            return None
        return tuple(int(v) for v in sz)

    def level_matrix(self, lev, what=0):
        sz = np.zeros(3, np.int32)
        if self._so.jxcpr_solver_level_sizes(self.h, lev, what, _ptr(sz)) < 0:
            return None
        n, m, nnz = (int(v) for v in sz)
        ia = np.zeros(n + 1, np.int32)
        ja = np.zeros(max(nnz, 1), np.int32)
        a = np.zeros(max(nnz, 1))
        if self._so.jxcpr_solver_level_matrix(self.h, lev, what, _ptr(ia), _ptr(ja), _ptr(a)) < 0:
            raise RuntimeError("level_matrix failed")
        return ia, ja[:nnz], a[:nnz], m

    def level_cf(self, lev, n):
        cf = np.zeros(n, np.int32)
        if self._so.jxcpr_solver_level_cf(self.h, lev, _ptr(cf)) < 0:
            return None
        return cf

    def decoupled_values(self, nnzb):
        a = np.zeros(nnzb * self.bs * self.bs)
        _lib.check(self._so.jxcpr_solver_decoupled_values(self.h, _ptr(a)))
        return a

    def cpr_apply(self, r):
        z = np.zeros(self.nb * self.bs)
        _lib.check(self._so.jxcpr_solver_cpr_apply(self.h, _ptr(np.ascontiguousarray(r, np.float64)), _ptr(z), 0))
        return z

    def stage2_sweep(self, b, x0):
        """One stage-2 sweep of the set-up preconditioner on A x = b from x0 (host arrays)."""
        x = np.array(x0, dtype=np.float64)
        _lib.check(self._so.jxcpr_solver_stage2_sweep(self.h, _ptr(np.ascontiguousarray(b, np.float64)), _ptr(x), 0))
        return x

    def vcycle(self, rp, xp=None):
        xp = np.zeros(self.nb) if xp is None else np.array(xp, dtype=np.float64)
        _lib.check(self._so.jxcpr_solver_vcycle(self.h, _ptr(np.ascontiguousarray(rp, np.float64)), _ptr(xp), 0))
        return xp

    def level_info(self, lev):
        sm, st = np.zeros(1, np.int32), np.zeros(1, np.int32)
        th, ch = np.zeros(1), np.zeros(6)
        if self._so.jxcpr_solver_level_info(self.h, lev, _ptr(sm), _ptr(st), _ptr(th), _ptr(ch)) < 0:
            return None
        return dict(smoother=int(sm[0]), storage=int(st[0]), theta=float(th[0]), cheb=ch[:3].copy(),
                    interval=(float(ch[3]), float(ch[4])), lambda_max=float(ch[5]))

    def level_features(self, lev):
        f = np.zeros(16, np.float32)
        n = self._so.jxcpr_solver_level_features(self.h, lev, _ptr(f))
        return None if n < 0 else f[:n].copy()

    def learned_status(self):
        o = np.zeros(5)
        _lib.check(self._so.jxcpr_solver_learned_status(self.h, _ptr(o)))
        return dict(learned_used=bool(o[0]), factor_learned=float(o[1]), factor_plain=float(o[2]),
                    bytes_learned=float(o[3]), bytes_plain=float(o[4]))

    def learned_fallbacks(self):
        """Solves in which the learned settings stalled and the plain preconditioner took over."""
        return int(self._so.jxcpr_solver_learned_fallbacks(self.h))

    def bilu_factors(self):
        """Block ILU(0) factors of stage2_solver_type 5: (la, ua, dinv) as flat host arrays."""
        sz = np.zeros(2, np.int64)
        _lib.check(self._so.jxcpr_solver_bilu_sizes(self.h, _ptr(sz)))
        bn = self.bs * self.bs
        la, ua, dinv = np.zeros(max(int(sz[0]), 1) * bn), np.zeros(max(int(sz[1]), 1) * bn), np.zeros(self.nb * bn)
        _lib.check(self._so.jxcpr_solver_bilu_factors(self.h, _ptr(la), _ptr(ua), _ptr(dinv)))
        return la[:int(sz[0]) * bn], ua[:int(sz[1]) * bn], dinv

    def bilu_apply(self, f):
        u = np.zeros(self.nb * self.bs)
        _lib.check(self._so.jxcpr_solver_bilu_apply(self.h, _ptr(np.ascontiguousarray(f, np.float64)), _ptr(u), 0))
        return u

    def level_stored_values(self, lev):
        """Level lev's operator values as the fast path stores them, in level_matrix's entry order."""
        nnz = self.level_sizes(lev, 0)[2]
        out = np.zeros(max(nnz, 1))
        _lib.check(self._so.jxcpr_solver_level_stored_values(self.h, lev, _ptr(out)))
        return out[:nnz]

    def bilu_levels(self):
        """bilu_exact 1: (lower levels per block row, upper levels per block row, #lower, #upper)."""
        lev_l, lev_u = np.zeros(self.nb, np.int32), np.zeros(self.nb, np.int32)
        cnt = np.zeros(2, np.int32)
        _lib.check(self._so.jxcpr_solver_bilu_levels(self.h, _ptr(lev_l), _ptr(lev_u), _ptr(cnt)))
        return lev_l, lev_u, int(cnt[0]), int(cnt[1])

    def close(self):
        if getattr(self, "h", None):
            self._so.jxcpr_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def setup_many(solvers, systems, threads=0):
    """jxcpr_solver_setup of solvers[k] with systems[k] (objects with ia, ja, a, block_size: host
    numpy arrays) on `threads` host threads (0: one per core)."""
    so = _lib.load()
    m = len(solvers)
    keep = [(np.ascontiguousarray(s.ia, np.int32), np.ascontiguousarray(s.ja, np.int32),
             np.ascontiguousarray(s.a, np.float64)) for s in systems]
    arr = lambda vals: (ctypes.c_void_p * m)(*vals)  # noqa: E731
    nb = np.array([len(k[0]) - 1 for k in keep], np.int32)
    bs = np.array([int(s.block_size) for s in systems], np.int32)
    nnzb = np.array([len(k[1]) for k in keep], np.int64)
    st = np.zeros(m, np.int32)
    rc = so.jxcpr_batch_setup(m, arr([G.h.value for G in solvers]), _ptr(nb), _ptr(bs), _ptr(nnzb),
                              arr([k[0].ctypes.data for k in keep]), arr([k[1].ctypes.data for k in keep]),
                              arr([k[2].ctypes.data for k in keep]), 0, int(threads), _ptr(st))
    _lib.check(rc)
    for G, s, k in zip(solvers, systems, keep):
        G.nb, G.bs = len(k[0]) - 1, int(s.block_size)
        G._keep = k
    return solvers


class CprGmresBatch:
    """Many set-up CprGmres solvers solved by one CUDA-graph launch.

    Each solver's whole GMRES solve is recorded as an independent branch of a
    single graph (graph_gmres mode: flexible GMRES, CGS2, device-side loop
    control).  The solvers must stay alive and unchanged while the batch is
    used.
    """

    def __init__(self, solvers):
        self._so = _lib.load()
        self.solvers = list(solvers)
        self.sizes = [s.nb * s.bs for s in self.solvers]
        arr = (ctypes.c_void_p * len(self.solvers))(*[s.h.value for s in self.solvers])
        h = ctypes.c_void_p()
        _lib.check(self._so.jxcpr_batch_create(ctypes.byref(h), len(self.solvers), arr))
        self.h = h

    def solve(self, bs, x0s=None, device=False):
        """Solves every system; returns dict of per-system arrays and the list of x.

        Host numpy arrays, or device pointers (ints) with device=True (then x0s
        are overwritten with the solutions)."""
        m = len(self.solvers)
        if device:
            bp = (ctypes.c_void_p * m)(*bs)
            xp = (ctypes.c_void_p * m)(*x0s)
            xs = list(x0s)
        else:
            bb = [np.ascontiguousarray(b, np.float64) for b in bs]
            xs = [np.zeros(n) if x0s is None else np.array(x0s[k], dtype=np.float64) for k, n in enumerate(self.sizes)]
            bp = (ctypes.c_void_p * m)(*[b.ctypes.data for b in bb])
            xp = (ctypes.c_void_p * m)(*[x.ctypes.data for x in xs])
        it = np.zeros(m, np.int32)
        rel = np.zeros(m)
        lat = np.zeros(m)
        fin = np.zeros(m)
        st = np.zeros(m, np.int32)
        rc = self._so.jxcpr_batch_solve(self.h, bp, xp, 1 if device else 0, _ptr(it), _ptr(rel), _ptr(lat),
                                        _ptr(fin), _ptr(st))
        if rc not in (0, STATUS_CONV):
            _lib.check(rc)
        return dict(x=xs, iterations=it, rel_residual=rel, latency_ms=lat, finish_ms=fin, status=st)

    def solve_ptrs(self, b_ptrs, x_ptrs, device):
        """Raw form of solve(): b_ptrs / x_ptrs are addresses (host with device=False, e.g. pinned
        buffers, or device); returns the per-system arrays only."""
        m = len(self.solvers)
        bp = (ctypes.c_void_p * m)(*b_ptrs)
        xp = (ctypes.c_void_p * m)(*x_ptrs)
        it = np.zeros(m, np.int32)
        rel = np.zeros(m)
        lat = np.zeros(m)
        fin = np.zeros(m)
        st = np.zeros(m, np.int32)
        rc = self._so.jxcpr_batch_solve(self.h, bp, xp, 1 if device else 0, _ptr(it), _ptr(rel), _ptr(lat),
                                        _ptr(fin), _ptr(st))
        if rc not in (0, STATUS_CONV):
            _lib.check(rc)
        return dict(iterations=it, rel_residual=rel, latency_ms=lat, finish_ms=fin, status=st)

    def last_ms(self):
        """Device time of the last solve: input copies, the graph launch and the output copies."""
        v = np.zeros(1)
        _lib.check(self._so.jxcpr_batch_last_ms(self.h, _ptr(v)))
        return float(v[0])

    def launch(self, stream_handle=0):
        _lib.check(self._so.jxcpr_batch_launch(self.h, ctypes.c_void_p(stream_handle)))

    def close(self):
        if getattr(self, "h", None):
            self._so.jxcpr_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
