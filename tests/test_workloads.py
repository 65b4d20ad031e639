"""Synthetic workload generators that tests and bench.py rely on (CPU)."""

import numpy as np

from hyperalignment_b200 import workloads as W


def test_duplicate_columns_to_fraction_exact_mask():
    w = W.small_case(seed=3, nv=642, nt=40, lo=20, hi=60)
    X = w.X.copy()
    mask = W.duplicate_columns_to_fraction(X, w.sls, 0.2, np.random.default_rng(0))
    frac = mask.mean()
    assert 0.2 <= frac < 0.45  # stops at the first pair that reaches the target
    for q in range(w.sls.count):
        sl = w.sls.indices[w.sls.offsets[q]:w.sls.offsets[q + 1]]
        has_dup = np.unique(X[:, sl], axis=1).shape[1] < sl.size
        assert has_dup == mask[q]


def test_rank_deficient_pair_fraction():
    w = W.rank_deficient_pair(0, nv=2562, nt=60, frac=0.1)
    m = w.extra["singular"]
    assert 0.1 <= m.mean() < 0.3
