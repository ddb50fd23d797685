"""The oracle's HMIS with the Ruge-Stueben first pass on row ranges (CPU).

One range is the whole-level pass that the hierarchy pins against the compiled
reference; with several ranges every point is still split into C or F, each
range's C points come from its own diagonal block of the strength pattern, and
the coarse grid stays within a few per cent of the single-pass one.
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
