"""Case-wise weighting and RF-GAP proximity on the GPU through the C ABI and
the pybind11 mirror, against the reference's own fit (oracle/_ref, use_casewise
/ use_rfgap) on forests it grew, and against the oracle (oracle/oracle.c) on
larger forests.  Every float and double sum runs in the reference's order, so
the comparisons are exact: weighted votes, OOB error / predictions /
probabilities, overall and local importance, the FP64 pair sums and the
finished float32 proximity, and the RF-GAP matrix."""
import warnings

import numpy as np
import pytest

from rfx_b200 import synth
from conftest import has_reference

pytestmark = pytest.mark.gpu

CASES = [(lambda: synth.mixed_cover(500, seed=61), 30, 7), (lambda: synth.gaussian_classes(400, 9, 3, seed=62), 25, 3)]


def _ref(case, **kw):
    from oracle import reference as ref

    gen, T, mtry = CASES[case]
    X, y = gen()
    y = np.unique(y, return_inverse=True)[1].astype(np.int32)
    cat = synth.detect_categorical(X)
    R = ref.fit_capture(X, y, cat, ntree=T, mtry=mtry, **kw)
    return X, y, R


def _upper(M):
    return M[np.triu_indices(M.shape[0])]


@pytest.mark.skipif(not has_reference(), reason="reference library not built")
@pytest.mark.parametrize("case", range(len(CASES)))
def test_casewise_cuda_matches_reference(built, case):
    from oracle import oracle as orc
    from rfx_b200 import abi

    X, y, R = _ref(case, use_casewise=True)
    f = R["forest"]
    O = orc.analyse(X, y, f, casewise=True, want_cw=True)
    ctx = abi.Context(0, use_casewise=True)
    ctx.load(f, X, y)
    q, nout = ctx.casewise_votes()
    assert np.array_equal(q, R["q_raw"]) and np.array_equal(nout, R["nout"])
    err, pred, proba = ctx.oob_summary()
    assert np.float32(err) == np.float32(R["oob_error"])
    assert np.array_equal(pred, R["oob_pred"]) and np.array_equal(proba, R["oob_proba"])
    avimp, sqsd, qimp, qimpm = ctx.varimp(True)
    assert np.array_equal(avimp, R["importances"]) and np.array_equal(sqsd, R["sqsd"])
    assert np.array_equal(qimp, R["qimp"])
    assert np.array_equal(ctx.localimp(qimp, qimpm), R["qimpm"])
    Sd = ctx.proximity_upper_f64()
    assert np.array_equal(Sd, O["Sd"])
    P = ctx.finishprox_f64(Sd, full=True)
    assert np.array_equal(P, R["prox"].astype(np.float32))
    # the integer entry points refuse the weighted context
    with pytest.raises(abi.RfxError):
        ctx.proximity_upper()
    ctx.close()


@pytest.mark.skipif(not has_reference(), reason="reference library not built")
@pytest.mark.parametrize("case", range(len(CASES)))
def test_rfgap_cuda_matches_reference(built, case):
    from rfx_b200 import abi

    X, y, R = _ref(case, use_rfgap=True)
    f = R["forest"]
    ctx = abi.Context(0)
    ctx.load(f, X, y)
    P = ctx.proximity_rfgap()
    assert np.array_equal(P, _upper(R["prox"]))
    ctx.close()


def test_weighted_paths_match_oracle_larger(built):
    """n = 5,000 (two column windows of the row kernel), 40 trees, against the
    oracle: case-wise votes, importance and FP64 sums; RF-GAP; and the
    unweighted FP64 sums equal to the INT32 counts."""
    from oracle import oracle as orc
    from rfx_b200 import abi

    X, y = synth.mixed_cover(5000, seed=63)
    y = np.unique(y, return_inverse=True)[1].astype(np.int32)
    f = abi.grow_forest(X, y, 40, 7, 1, nclass=int(y.max()) + 1, cat=synth.detect_categorical(X))
    O = orc.analyse(X, y, f, casewise=True, want_cw=True, want_leaf=True)
    ctx = abi.Context(0, use_casewise=True)
    ctx.load(f, X, y)
    q, _ = ctx.casewise_votes()
    assert np.array_equal(q, O["q_raw"])
    avimp, sqsd, qimp, qimpm = ctx.varimp(True)
    assert np.array_equal(avimp, O["avimp"]) and np.array_equal(qimpm, O["qimpm"])
    assert np.array_equal(ctx.proximity_upper_f64(), O["Sd"])
    ctx.close()
    ctx = abi.Context(0)
    ctx.load(f, X, y)
    P = ctx.proximity_rfgap()
    assert np.array_equal(P, _upper(orc.rfgap(f.nin, O["leaf"])))
    S = ctx.proximity_upper()
    assert np.array_equal(ctx.proximity_upper_f64(), S.astype(np.float64))
    ctx.close()


@pytest.mark.skipif(not has_reference(), reason="reference library not built")
def test_pybind_casewise_and_rfgap_match_reference(built):
    from oracle import reference as ref
    from rfx_b200 import _rfx as rfx

    X, y = synth.mixed_cover(450, seed=64)
    y = np.unique(y, return_inverse=True)[1].astype(np.int32)
    cat = synth.detect_categorical(X)
    n, p = X.shape
    for kw in (dict(use_casewise=True), dict(use_rfgap=True)):
        R = ref.fit_capture(X, y, cat, ntree=20, mtry=7, **kw)
        m = rfx.RandomForestClassifier(nsample=n, ntree=20, mdim=p, mtry=7, compute_proximity=True,
                                       compute_importance=True, compute_local_importance=True, use_gpu=True,
                                       show_progress=False, **kw)
        m.fit(X, y)
        assert np.float32(m.get_oob_error()) == np.float32(R["oob_error"])
        assert np.array_equal(m.feature_importances_(), R["importances"])
        assert np.array_equal(m.get_local_importance(), R["qimpm"])
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            P = m.get_proximity_matrix()
        assert np.array_equal(P, R["prox"].astype(np.float32)), kw
        m.cleanup()
