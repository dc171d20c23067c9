"""CUDA path (through the C ABI) against the oracle on forests and inputs that
grown forests rarely produce: single-leaf trees, a tree with no OOB sample
(its importance is the reference's 0/0 = NaN), a tree with no in-bag sample,
NaN in continuous features, and categorical values outside 0..cat-1.

Where a categorical value rounds outside 0..maxcat-1, the reference's
permuted walk stops without a vote and keeps a value that depends on its
OpenMP thread count; the CUDA path reports that with an error instead of a
number, and everything else (routing, votes, pair counts) still matches."""
import numpy as np
import pytest

from rfx_b200 import synth
from conftest import single_leaf_tree

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def grown(built):
    from rfx_b200 import abi

    X, y = synth.mixed_cover(700, seed=23)
    y = np.unique(y, return_inverse=True)[1].astype(np.int32)
    f = abi.grow_forest(X, y, 16, 7, 1, nclass=int(y.max()) + 1, cat=synth.detect_categorical(X))
    return X, y, f


def _no_oob(f, t):
    g = f.subset(range(f.ntree))
    g.nin[t] = np.maximum(g.nin[t], 1)
    return g


def _no_inbag(f, t):
    g = f.subset(range(f.ntree))
    g.nin[t] = 0
    return g


def _set_entries(X, f, cols_of, value, seed, count=80):
    rng = np.random.default_rng(seed)
    X2 = X.copy()
    cols = np.flatnonzero(cols_of(f.cat))
    X2[rng.choice(f.n, size=count, replace=False), rng.choice(cols, size=count)] = np.float32(value)
    return X2


CASES = {
    "single_leaf_trees": lambda X, y, f: (X, single_leaf_tree(single_leaf_tree(f, 0, 0), 7, f.nclass - 1)),
    "tree_without_oob": lambda X, y, f: (X, _no_oob(f, 3)),
    "tree_without_inbag": lambda X, y, f: (X, _no_inbag(f, 2)),
    "nan_continuous": lambda X, y, f: (_set_entries(X, f, lambda c: c == 1, np.nan, 5), f),
}
# values whose (int)(x + 0.5f) stays in 0..maxcat-1: every permuted walk ends in a leaf
for _v in (-1.0, -0.4, 0.49, 0.5, 1.5, 2.0, 9.0):
    CASES[f"categorical_{_v}"] = (lambda v: lambda X, y, f: (_set_entries(X, f, lambda c: c > 1, v, 7), f))(_v)


def _check(X, y, f, varimp_may_refuse=False):
    from oracle import oracle as orc
    from rfx_b200 import abi

    O = orc.analyse(X, y, f, want_leaf=True)
    ctx = abi.Context(0)
    try:
        ctx.load(f, X, y)
        leaf = np.zeros((f.ntree, f.n), np.int32)
        q, nout, _ = ctx.route_oob(leaf=leaf)
        assert np.array_equal(q.astype(np.float32), O["q_raw"])
        assert np.array_equal(nout, O["nout"])
        assert np.array_equal(leaf, O["leaf"])
        assert np.array_equal(ctx.proximity_upper(), O["S"])
        try:
            avimp, sqsd, qimp, qimpm = ctx.varimp(impn=True)
        except abi.RfxError as e:
            assert varimp_may_refuse and "cpu_testreeimp" in str(e)
        else:
            assert np.array_equal(avimp, O["avimp"], equal_nan=True)
            assert np.array_equal(sqsd, O["sqsd"], equal_nan=True)
            assert np.array_equal(qimp, O["qimp"])
            assert np.array_equal(qimpm, O["qimpm"])
        votes = ctx.predict_votes(X)
        assert np.array_equal(votes, orc.predict(X, f)[0])
        # the context stays usable after a refused call
        assert np.array_equal(ctx.proximity_upper(), O["S"])
    finally:
        ctx.close()
    return O


@pytest.mark.parametrize("name", list(CASES))
def test_edge_case_matches_oracle(grown, name):
    X, y, f = grown
    X2, g = CASES[name](X, y, f)
    O = _check(X2, y, g)
    if name == "tree_without_oob":
        assert np.isnan(O["avimp"]).any()


@pytest.mark.parametrize("value", [-2.0, 9.6, 12.0])
def test_categorical_value_beyond_maxcat(grown, value):
    X, y, f = grown
    _check(_set_entries(X, f, lambda c: c > 1, value, 11), y, f, varimp_may_refuse=True)
