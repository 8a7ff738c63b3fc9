"""The parallel-column groups the engine re-expresses before a PDHG / PDLP
solve (nir_pdhg_parallel_groups, host code of libnir_pdhg.so; no GPU)."""
import numpy as np
import pytest

from nirnaya_b200 import lp as L
from nirnaya_b200 import pdhg


def _lp_from_columns(cols, m):
    """An LP with the given columns (lists of (row, value)), 0 <= x <= 10."""
    start, idx, val = [0], [], []
    for c in cols:
        for r, v in c:
            idx.append(r)
            val.append(v)
        start.append(len(idx))
    n = len(cols)
    return L.LP(m, n, np.array(start, np.int64), np.array(idx, np.int32), np.array(val, float), np.ones(n),
                np.zeros(n), np.full(n, 10.0), np.zeros(m), np.ones(m))


def test_badly_scaled_duplicates_form_one_group_each():
    lp = L.generate(L.BADLY_SCALED, 1, m=500, n=1200, target_nnz=10000)
    rep, lam, groups = pdhg.parallel_groups(lp)
    nb = lp.ncol // 2
    assert groups == nb
    assert np.array_equal(rep[:nb], np.full(nb, -1))
    assert np.array_equal(rep[nb:], np.arange(nb))
    assert np.max(np.abs(lam[nb:] - 1.0)) < 1e-7  # duplicated with a 1e-9 perturbation


def test_random_lp_has_no_groups():
    _, _, groups = pdhg.parallel_groups(L.generate(L.RANDOM_EQ, 3, m=300, n=700))
    assert groups == 0


def test_groups_proportions_patterns_and_tolerance():
    a = [(0, 1.0), (2, -3.0), (5, 0.5)]
    cols = [
        a,                                               # 0: representative
        [(0, -2.0), (2, 6.0), (5, -1.0)],                # 1: -2 x column 0
        [(0, 1.0), (2, -3.0)],                           # 2: another pattern
        [(0, 3.0), (2, -9.0), (5, 1.5 * (1 + 1e-7))],    # 3: 3 x column 0, eps within 1e-6
        [(0, 1.0), (2, -3.0), (5, 0.6)],                 # 4: same pattern, not parallel
        [(1, 4.0), (4, 1.0)],                            # 5: representative of its own
        [(1, 8.0), (4, 2.0)],                            # 6: 2 x column 5
        [],                                              # 7: empty: never grouped
        [],                                              # 8
        [(3, 1.0)],                                      # 9: single entries: never grouped
        [(3, 5.0)],                                      # 10
    ]
    rep, lam, groups = pdhg.parallel_groups(_lp_from_columns(cols, 6))
    assert groups == 2
    assert rep.tolist() == [-1, 0, -1, 0, -1, -1, 5, -1, -1, -1, -1]
    assert lam[1] == -2.0 and lam[3] == pytest.approx(3.0, rel=1e-12) and lam[6] == 2.0


def test_power_law_lp_has_no_groups():
    # its coincidental pairs are single-entry columns of one row
    _, _, groups = pdhg.parallel_groups(L.generate(L.ZIPF, 1, m=20000, n=50000, target_nnz=500000))
    assert groups == 0


def test_rejects_a_malformed_lp():
    lp = _lp_from_columns([[(0, 1.0)], [(3, 1.0)]], 2)  # row index out of range
    with pytest.raises(RuntimeError):
        pdhg.parallel_groups(lp)
