"""The oracle's HMIS with the Ruge-Stueben first pass on row ranges (CPU).

One range is the whole-level pass.  The first pass itself is pinned to the
compiled reference (jxf_PAMGCoarsenRuge, coarsen_type 10) on every level's
strength pattern, and the ranged pass to the reference run on each range's
diagonal block -- what each process of a distributed run computes -- wherever
no row's strong connections all leave its range (for such rows the ranged pass
follows par_coarsen_ruge.c:261: SF_PT only for a row with no strong connection
at all).  With several ranges every point is still split into C or F and the
coarse grid stays within a few per cent of the single-pass one.
"""
import numpy as np
import pytest

import oracle
from jxpamg_all_b200 import synth


def level0(name):
    s = synth.config_system(name)
    a, _ = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    C = oracle.OracleCPR(s.ia, s.ja, a, s.block_size)
    ia, ja, av, _ = C.level_matrix(0, 0)
    return C, ia, ja, av


def test_one_range_is_the_whole_level_pass():
    C, ia, ja, a = level0("c0")
    n = len(ia) - 1
    cf = C.level_cf(0, n)
    assert np.array_equal(oracle.hmis_cf(ia, ja, a), cf)
    assert np.array_equal(oracle.hmis_cf(ia, ja, a, range_rows=n), cf)
    assert np.array_equal(oracle.hmis_cf(ia, ja, a, range_rows=n // 2 + 1), cf)  # n / rows < 2: one range


@pytest.mark.parametrize("rows", [500, 1000, 2667])
def test_ranges_split_every_point(rows):
    C, ia, ja, a = level0("c0")
    n = len(ia) - 1
    cf = oracle.hmis_cf(ia, ja, a, range_rows=rows)
    cf1 = C.level_cf(0, n)
    assert set(np.unique(cf)) <= {-1, 1}
    nc, nc1 = int((cf == 1).sum()), int((cf1 == 1).sum())
    assert abs(nc - nc1) <= 0.1 * nc1, (nc, nc1)
    # away from the range borders the splitting is the whole-level one in most places
    assert (cf == cf1).mean() >= 0.6


def test_ranges_only_change_with_range_count():
    _, ia, ja, a = level0("c0")
    n = len(ia) - 1
    # n // rows ranges of near-equal size: row counts giving the same number of ranges agree
    assert np.array_equal(oracle.hmis_cf(ia, ja, a, range_rows=n // 4), oracle.hmis_cf(ia, ja, a, range_rows=n // 4 - 100))


def _diag_block(sia, sja, r0, r1):
    """The strength pattern of rows r0..r1 restricted to the same columns (shifted to 0)."""
    li, lj, cross_only = [0], [], 0
    for i in range(r0, r1):
        row = [j - r0 for j in sja[sia[i]:sia[i + 1]] if r0 <= j < r1]
        cross_only += (not row) and sia[i + 1] > sia[i]
        lj += row
        li.append(len(lj))
    return np.array(li, np.int32), np.array(lj, np.int32), cross_only


@pytest.mark.ref
@pytest.mark.parametrize("name", ["c0", "small", "tiny3"])
def test_first_pass_pinned_to_reference(name):
    """The restated first pass equals the reference's (jxf_PAMGCoarsenRuge, coarsen_type 10) on
    every level's strength pattern."""
    s = synth.config_system(name)
    a, _ = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    C = oracle.OracleCPR(s.ia, s.ja, a, s.block_size)
    for lev in range(C.num_levels() - 1):
        ia, ja, av, _ = C.level_matrix(lev, 0)
        sia, sja = oracle.strength(ia, ja, av)
        assert np.array_equal(oracle.rs_first_pass(sia, sja), oracle.ref_rs_first_pass(sia, sja)), lev


@pytest.mark.ref
@pytest.mark.parametrize("name,ranges", [("c0", 2), ("c0", 3), ("c0", 5), ("small", 3), ("small", 5)])
def test_ranged_first_pass_pinned_to_reference(name, ranges):
    """Where no row's strong connections all leave its range, the ranged pass equals the
    reference's first pass run on each range's diagonal block (what each process of a
    distributed run computes)."""
    _, ia, ja, av = level0(name)
    sia, sja = oracle.strength(ia, ja, av)
    n = len(sia) - 1
    rows = n // ranges
    ours = oracle.rs_first_pass(sia, sja, range_rows=rows)
    nr = n // rows
    for r in range(nr):
        r0, r1 = n * r // nr, n * (r + 1) // nr
        li, lj, cross_only = _diag_block(sia, sja, r0, r1)
        assert cross_only == 0
        assert np.array_equal(ours[r0:r1], oracle.ref_rs_first_pass(li, lj)), r


def test_rows_strong_only_across_ranges_are_not_special_fine():
    """A row whose strong connections all lie in other ranges is still split (SF_PT only for a row
    without any strong connection, par_coarsen_ruge.c:261)."""
    s = synth.config_system("c0")
    a, _ = oracle.bsr_decouple(s.ia, s.ja, s.a, s.block_size, s.b, 1)
    C = oracle.OracleCPR(s.ia, s.ja, a, s.block_size)
    ia, ja, av, _ = C.level_matrix(1, 0)
    sia, sja = oracle.strength(ia, ja, av)
    n = len(sia) - 1
    rows = n // 3
    cf = oracle.rs_first_pass(sia, sja, range_rows=rows)
    seen = 0
    for r in range(3):
        r0, r1 = n * r // 3, n * (r + 1) // 3
        for i in range(r0, r1):
            local = [j for j in sja[sia[i]:sia[i + 1]] if r0 <= j < r1]
            if not local and sia[i + 1] > sia[i]:
                seen += 1
                assert cf[i] != -3, i
    assert seen >= 1
    assert np.all((cf == -3) == (np.diff(sia) == 0))
