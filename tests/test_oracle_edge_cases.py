"""The oracle against the reference's own CPU code on edge cases that grown
forests rarely reach: single-leaf trees, trees with no OOB sample (the
reference's 0/0 importance), trees with no in-bag sample, NaN feature values,
and categorical values outside 0..cat-1 (negative, too large, fractional).

Each case starts from a forest the reference grew and then changes the forest
or the analysed X; both implementations analyse the same (forest, X).

A categorical value that rounds outside 0..maxcat-1 makes cpu_testreeimp
(src/rf_varimp.cpp:84-100) stop without a vote, and the permuted vote of that
sample is then whatever the per-thread jvr buffer held from the previous
feature the same OpenMP thread processed (src/rf_varimp.cpp:184-190).  That
depends on how many threads the reference ran with; the oracle restates the
one-thread order, so those cases run the reference on one thread.  The CUDA
path refuses such inputs with an error instead of picking a thread count.
"""
import contextlib

import numpy as np
import pytest

from rfx_b200 import synth
from conftest import has_reference, single_leaf_tree

pytestmark = pytest.mark.skipif(not has_reference(), reason="reference library not built")


@contextlib.contextmanager
def _reference_threads(k):
    from oracle import reference as ref

    before = ref.set_threads(0)
    ref.set_threads(k)
    try:
        yield
    finally:
        ref.set_threads(before)


@pytest.fixture(scope="module")
def grown(built):
    from oracle import reference as ref

    X, y = synth.mixed_cover(260, seed=17)
    y = np.unique(y, return_inverse=True)[1].astype(np.int32)
    cat = synth.detect_categorical(X)
    f = ref.grow_forest(X, y, 12, 7, 1, cat=cat)
    return X, y, f


def _compare(X, y, f, threads=None):
    """Votes, nout, leaf ids, importances and raw pair counts, bit for bit
    (NaN where the reference divides 0 by 0 counts as equal)."""
    from oracle import oracle as orc, reference as ref

    with _reference_threads(threads) if threads else contextlib.nullcontext():
        R = ref.analyse_trees(X, y, f, do_prox=True, want_leaf=True)
    O = orc.analyse(X, y, f, want_leaf=True)
    n = f.n
    assert np.array_equal(O["q_raw"].reshape(-1), R["q"])
    assert np.array_equal(O["nout"], R["nout"])
    assert np.array_equal(O["leaf"], R["leaf"])
    for k in ("qimp", "qimpm", "avimp", "sqsd"):
        assert np.array_equal(O[k], R[k], equal_nan=True), k
    # the reference adds 1 to prox[i + j*n] for OOB i and in-bag j in one leaf
    C = R["prox"].reshape(n, n).T
    assert np.array_equal(orc.upper_to_full(O["S"], n).astype(np.float64), C + C.T)
    return O, R


def test_single_leaf_trees(grown):
    X, y, f = grown
    g = single_leaf_tree(single_leaf_tree(f, 0, 0), 5, f.nclass - 1)
    _compare(X, y, g)


def test_tree_without_oob_samples(grown):
    X, y, f = grown
    g = f.subset(range(f.ntree))
    g.nin[3] = np.maximum(g.nin[3], 1)
    O, _ = _compare(X, y, g)
    assert np.isnan(O["avimp"]).any()      # features split on in tree 3 get 0/0


def test_tree_without_inbag_samples(grown):
    X, y, f = grown
    g = f.subset(range(f.ntree))
    g.nin[2] = 0
    _compare(X, y, g)


def test_nan_in_continuous_features(grown):
    X, y, f = grown
    rng = np.random.default_rng(5)
    X2 = X.copy()
    cont = np.flatnonzero(f.cat == 1)
    rows = rng.choice(f.n, size=40, replace=False)
    X2[rows, rng.choice(cont, size=40)] = np.nan
    _compare(X2, y, f)


@pytest.mark.parametrize("value", [-1.0, -0.6, -0.4, 0.49, 0.5, 1.5, 2.0, 9.0, 9.6, 12.0])
def test_categorical_values_out_of_range(grown, value):
    X, y, f = grown
    rng = np.random.default_rng(int(value * 10) + 100)
    X2 = X.copy()
    catcols = np.flatnonzero(f.cat > 1)
    rows = rng.choice(f.n, size=60, replace=False)
    X2[rows, rng.choice(catcols, size=60)] = np.float32(value)
    _compare(X2, y, f, threads=1)


@pytest.mark.parametrize("seed", [0, 1])
def test_nonzero_catgoleft(grown, seed):
    """Random go-left tables: the three walks index them differently
    (testreebag by the truncated value, find_terminal_node by the 1-based
    rounded value, testreeimp by the rounded value), and the oracle follows
    each as the reference does."""
    X, y, f = grown
    g = f.subset(range(f.ntree))
    rng = np.random.default_rng(seed)
    g.catgoleft = rng.integers(0, 2, size=g.total_nodes * g.maxcat).astype(np.int32)
    O, _ = _compare(X, y, g, threads=1)
    assert O["S"].any()


@pytest.mark.parametrize("seed", [0, 1])
def test_predict_with_catgoleft_and_invalid_codes(grown, seed):
    """predict / predict_proba through random go-left tables, with test codes
    outside 1..cat (the reference votes 0 for those)."""
    from oracle import oracle as orc, reference as ref

    X, y, f = grown
    g = f.subset(range(f.ntree))
    rng = np.random.default_rng(seed)
    g.catgoleft = rng.integers(0, 2, size=g.total_nodes * g.maxcat).astype(np.int32)
    Xt = (X[:90] + rng.normal(0, 0.4, size=X[:90].shape)).astype(np.float32)
    Xt[:, g.cat > 1] = np.round(Xt[:, g.cat > 1] * 2.0)  # codes -2..4, some outside 1..cat
    _, pred, proba = orc.predict(Xt, g)
    rp, rpr = ref.predict(Xt, g)
    assert np.array_equal(pred, rp)
    assert np.array_equal(proba, rpr)


def test_status2_nodes(grown):
    """Created-but-unsplit nodes (status 2, children 0): testreebag stops on
    them, find_terminal_node walks through them back to the root, and the
    permuted walks of cpu_testreeimp pass through them without a vote (the
    one-thread stale order, as above)."""
    X, y, f = grown
    g = f.subset(range(f.ntree))
    rng = np.random.default_rng(4)
    for t in range(g.ntree):
        o = g.offs[t]
        leaves = np.flatnonzero(g.nodestatus[o:g.offs[t + 1]] == -1)
        pick = o + rng.choice(leaves, size=max(1, leaves.size // 4), replace=False)
        g.nodestatus[pick] = 2
        g.treemap[2 * pick] = 0
        g.treemap[2 * pick + 1] = 0
    _compare(X, y, g, threads=1)
