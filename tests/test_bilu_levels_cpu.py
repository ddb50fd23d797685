"""Level schedule of the exact block ILU(0) (oracle restatement, no reference needed): levels
respect every dependency and are the longest-path depths of the lower / upper DAGs; the exact
factors satisfy A = (I + L)(D + U) on A's pattern."""
import numpy as np
import pytest

import oracle


@pytest.mark.parametrize("name", ["tiny", "small", "tiny3", "c0"])
def test_levels_are_longest_paths(systems, name):
    s = systems(name)
    lia, lja, uia, uja = oracle.bilu_pattern(s.ia, s.ja)
    lev_l, lev_u, nl, nu = oracle.bilu_levels(s.ia, s.ja)
    nb = s.num_block_rows
    for r in range(nb):
        deps = lja[lia[r]:lia[r + 1]]
        assert lev_l[r] == (1 + lev_l[deps].max() if len(deps) else 0)
        deps = uja[uia[r]:uia[r + 1]]
        assert lev_u[r] == (1 + lev_u[deps].max() if len(deps) else 0)
    assert nl == lev_l.max() + 1 and nu == lev_u.max() + 1


@pytest.mark.parametrize("name", ["small", "tiny3"])
def test_exact_factors_reproduce_a_on_its_pattern(systems, name):
    s = systems(name)
    bs = s.block_size
    a, _ = oracle.bsr_decouple(s.ia, s.ja, s.a, bs, s.b, 1)
    F = oracle.bilu_setup_exact(s.ia, s.ja, a, bs)
    nb = s.num_block_rows
    L = {}
    U = {}
    D = {}
    for r in range(nb):
        for k in range(F["lia"][r], F["lia"][r + 1]):
            L[(r, int(F["lja"][k]))] = F["la"][k * bs * bs:(k + 1) * bs * bs].reshape(bs, bs)
        for k in range(F["uia"][r], F["uia"][r + 1]):
            U[(r, int(F["uja"][k]))] = F["ua"][k * bs * bs:(k + 1) * bs * bs].reshape(bs, bs)
        D[r] = np.linalg.inv(F["dinv"][r * bs * bs:(r + 1) * bs * bs].reshape(bs, bs))
    A = a.reshape(-1, bs, bs)
    worst = 0.0
    for r in range(nb):
        for jj in range(s.ia[r], s.ia[r + 1]):
            c = int(s.ja[jj])
            # ((I + L)(D + U))_rc = sum_k (I + L)_rk (D + U)_kc
            acc = np.zeros((bs, bs))
            for k in range(min(r, c) + 1):
                left = np.eye(bs) if k == r else L.get((r, k))
                if left is None:
                    continue
                right = D[k] if k == c else U.get((k, c))
                if right is None:
                    continue
                acc += left @ right
            worst = max(worst, np.abs(acc - A[jj]).max() / max(1.0, np.abs(A[jj]).max()))
    assert worst < 1e-10
