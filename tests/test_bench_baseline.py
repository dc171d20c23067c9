"""bench.py's CPU legs on small cases: the forest's pair-update count (the
metric's unit) equals the sum of the oracle's pair counts, and the sampled
per-tree runner accumulates into one array exactly what a whole-forest
analysis does."""
import os
import sys

import numpy as np

from rfx_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _forest(n=600, T=24):
    from rfx_b200 import abi

    X, y = synth.mixed_cover(n, seed=31)
    y = np.unique(y, return_inverse=True)[1].astype(np.int32)
    f = abi.grow_forest(X, y, T, 7, 1, nclass=int(y.max()) + 1, cat=synth.detect_categorical(X))
    return X, y, f


def test_forest_pair_updates_is_the_sum_of_pair_counts(built):
    sys.path.insert(0, ROOT)
    import bench
    from oracle import oracle as orc

    X, y, f = _forest()
    S = orc.analyse(X, y, f, do_imp=False, impn=False, do_prox=True)["S"]
    assert bench.forest_pair_updates(X, y, f) == int(S.astype(np.int64).sum())


def test_sampled_trees_accumulate_the_forest_counts(built):
    sys.path.insert(0, ROOT)
    import bench
    from oracle import oracle as orc

    X, y, f = _forest(n=300, T=10)
    run = bench.CpuTrees(X, y, f)
    for k in range(f.ntree):
        assert run.tree_seconds(k) > 0.0
    assert sorted(run.order.tolist()) == list(range(f.ntree))
    S = orc.analyse(X, y, f, do_imp=False, impn=False, do_prox=True)["S"]
    assert np.array_equal(run.S, S)
    v, info = bench.cpu_baseline_run(X, y, f, budget_s=0.0, min_trees=3)
    assert v > 0 and info["trees"] == 3
