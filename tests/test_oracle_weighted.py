"""The oracle's case-wise weighting and RF-GAP proximity against the
reference's own fit (oracle/_ref) with use_casewise=True / use_rfgap=True on
forests the reference grew:

* case-wise: OOB votes weighted by tnodewt (the mean bootstrap multiplicity
  of a terminal node's in-bag samples), the weighted OOB error, overall and
  local importance with tnodewt weights, and the FP64 proximity sums with
  weights nin / nodesize through cpu_finishprox — bit for bit;
* RF-GAP: pGAP from the reference's per-tree node ids and multiplicities,
  symmetrised — bit for bit.
"""
import numpy as np
import pytest

from rfx_b200 import synth
from conftest import has_reference

pytestmark = pytest.mark.skipif(not has_reference(), reason="reference library not built")


def _case(gen, T, mtry, **kw):
    from oracle import reference as ref

    X, y = gen()
    y = np.unique(y, return_inverse=True)[1].astype(np.int32)
    cat = synth.detect_categorical(X)
    R = ref.fit_capture(X, y, cat, ntree=T, mtry=mtry, **kw)
    return X, y, R


CASES = [(lambda: synth.mixed_cover(500, seed=61), 30, 7), (lambda: synth.gaussian_classes(400, 9, 3, seed=62), 25, 3)]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_casewise_matches_reference(built, case):
    from oracle import oracle as orc

    gen, T, mtry = CASES[case]
    X, y, R = _case(gen, T, mtry, use_casewise=True)
    f = R["forest"]
    O = orc.analyse(X, y, f, casewise=True, want_cw=True)
    assert np.array_equal(O["q_raw"], R["q_raw"])
    assert np.array_equal(O["nout"], R["nout"])
    err, pred, proba = orc.oob_summary(O["q_raw"], O["nout"], y)
    assert np.float32(err) == np.float32(R["oob_error"])
    assert np.array_equal(pred, R["oob_pred"]) and np.array_equal(proba, R["oob_proba"])
    assert np.array_equal(O["avimp"], R["importances"]) and np.array_equal(O["sqsd"], R["sqsd"])
    assert np.array_equal(O["qimp"], R["qimp"])
    assert np.array_equal(orc.localimp(O["qimp"], O["qimpm"], f.n, f.p, f.ntree), R["qimpm"])
    P = orc.finishprox_f64(O["Sd"], O["nout"], full=True)
    assert np.array_equal(P, R["prox"].astype(np.float32))
    # the casewise sums differ from the plain counts
    O0 = orc.analyse(X, y, f)
    assert not np.array_equal(O0["q_raw"], O["q_raw"])


@pytest.mark.parametrize("case", range(len(CASES)))
def test_rfgap_matches_reference(built, case):
    from oracle import oracle as orc

    gen, T, mtry = CASES[case]
    X, y, R = _case(gen, T, mtry, use_rfgap=True)
    f = R["forest"]
    O = orc.analyse(X, y, f, do_imp=False, do_prox=False, want_leaf=True)
    P = orc.rfgap(f.nin, O["leaf"])
    assert np.array_equal(P, R["prox"])
    assert np.allclose(P.sum(), f.n)  # each pGAP row sums to 1
