"""The throughput path's stage-2 order, on the CPU (no GPU needed).

The reference's stage 2 sweeps the block rows in natural order
(jxf_ParBSRHGSRelax, par_relax_bsr.c:193-573).  A plain multicolour order
loses the coupling along the grid's fastest index that this sweep carries on
the upwinded Jacobians (57 GMRES iterations on the 1.12M-cell system instead
of the reference's 51); the chunk order keeps it: chunks of consecutive rows
visited in natural order, the chunks coloured for parallelism.

* the library's host ordering (jxcpr_stage2_chunk_order) equals the oracle's
  restatement and is a valid schedule: no two coupled chunks share a colour,
  chunks stay whole and aligned inside the 32-row slices;
* with the oracle's natural-order V-cycle, the chunk-ordered stage 2 keeps the
  iteration count of the natural-order one within +-10 %.
"""
import ctypes

import numpy as np
import pytest

import oracle
from jxpamg_all_b200 import lib


def product_order(ia, ja, chunk):
    so = lib.load()
    ia = np.ascontiguousarray(ia, np.int32)
    ja = np.ascontiguousarray(ja, np.int32)
    nb = len(ia) - 1
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    n = so.jxcpr_stage2_chunk_order(nb, P(ia), P(ja), chunk, None, 0, None, 0)
    assert n >= 0
    order = np.zeros(max(n, 1), np.int32)
    seg = np.zeros(nb + 2, np.int32)
    assert so.jxcpr_stage2_chunk_order(nb, P(ia), P(ja), chunk, P(order), n, P(seg), len(seg)) == n
    nseg = 1 + int(np.count_nonzero(seg[1:]))
    return order[:n], seg[:nseg]


def random_pattern(nb, per_row, seed):
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(nb):
        cols = set(rng.integers(0, nb, per_row).tolist()) - {i}
        rows.append([i] + sorted(cols))
    ia = np.zeros(nb + 1, np.int32)
    ia[1:] = np.cumsum([len(r) for r in rows])
    ja = np.concatenate([np.array(r, np.int32) for r in rows])
    return ia, ja


CASES = ["small", "c0", "tiny3", "random"]


def pattern(systems, name):
    if name == "random":
        return random_pattern(1003, 6, 5)  # not a multiple of the chunk length, irregular coupling
    s = systems(name)
    return s.ia, s.ja


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("chunk", [4, 8, 16])
def test_chunk_order_matches_oracle_and_is_a_schedule(systems, name, chunk):
    ia, ja = pattern(systems, name)
    nb = len(ia) - 1
    order, seg = product_order(ia, ja, chunk)
    colour, ncol = oracle.chunk_colour(ia, ja, chunk)
    assert len(seg) == ncol + 1 and seg[0] == 0 and seg[-1] == len(order)
    assert np.all(seg % 32 == 0)
    # every row once; each stored row's segment is its chunk's oracle colour
    live = order >= 0
    assert np.array_equal(np.sort(order[live]), np.arange(nb))
    for c in range(ncol):
        part = order[seg[c]:seg[c + 1]]
        assert np.all(colour[part[part >= 0]] == c)
        # chunks whole and aligned: slot t holds row chunk_start + t % chunk
        for t in range(0, len(part), chunk):
            blk = part[t:t + chunk]
            rows = blk[blk >= 0]
            if len(rows):
                base = rows[0] - rows[0] % chunk
                assert base % chunk == 0
                expect = np.arange(base, base + chunk)
                assert np.array_equal(blk[blk >= 0], expect[expect < nb][:len(rows)])
                assert np.array_equal(np.nonzero(blk >= 0)[0], np.arange(len(rows)))
    # a valid schedule: coupled rows in different chunks have different colours (symmetrised)
    r = np.repeat(np.arange(nb), np.diff(ia))
    other = (r // chunk) != (ja // chunk)
    assert np.all(colour[r[other]] != colour[ja[other]])


@pytest.mark.parametrize("name", ["small", "c0", "tiny3"])
def test_chunk_order_keeps_the_natural_iteration_count(systems, name):
    s = systems(name)
    a, b = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    its = {}
    for chunk in (0, 8):
        O = oracle.OracleCPR(s.ia, s.ja, a, s.block_size, stage2_chunk=chunk)
        its[chunk] = oracle.gmres(s.ia, s.ja, a, s.block_size, b, tol=1e-6, max_iter=300, cpr=O)["iters"]
    assert abs(its[8] - its[0]) <= 0.10 * its[0], its


def test_chunk_order_rejects_bad_chunk():
    so = lib.load()
    ia = np.array([0, 1], np.int32)
    ja = np.array([0], np.int32)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    assert so.jxcpr_stage2_chunk_order(1, P(ia), P(ja), 5, None, 0, None, 0) == -4
