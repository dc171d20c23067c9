"""Committed golden fixtures (tests/golden/*.npz, made by
tests/golden/make_golden.py from the reference's own CPU code) against the
oracle (CPU) and the CUDA path through the C ABI (GPU)."""
import glob
import os

import numpy as np
import pytest

from conftest import ROOT
from rfx_b200.forest import Forest

GOLDEN = os.path.join(ROOT, "tests", "golden")
# the fixtures with the full proximity matrix; config1_n2000_t500 (digests of
# the matrix instead) is checked by tests/test_config_parity.py
FILES = sorted(f for f in glob.glob(os.path.join(GOLDEN, "*.npz"))
               if not f.endswith(("permobmr.npz", "config1_n2000_t500.npz")))


def load(path):
    z = np.load(path)
    n, p = z["X"].shape
    nnode = z["nnode"]
    offs = np.zeros(nnode.size + 1, np.int64)
    offs[1:] = np.cumsum(nnode)
    f = Forest(n, p, int(z["nclass"]), int(z["maxcat"]), nnode, offs, z["nodestatus"], z["bestvar"],
               z["xbestsplit"], z["treemap"], z["nodeclass"], z["nin"], z["cat"])
    return z, f


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f)[:-4] for f in FILES])
def test_oracle_matches_golden(built, path):
    from oracle import oracle as orc

    z, f = load(path)
    O = orc.analyse(z["X"], z["y"], f)
    assert np.array_equal(O["q_raw"], z["q_raw"])
    assert np.array_equal(O["nout"], z["nout"])
    assert np.array_equal(O["avimp"], z["importances"])
    assert np.array_equal(O["sqsd"], z["sqsd"])
    assert np.array_equal(O["qimp"], z["qimp"])
    assert np.array_equal(orc.localimp(O["qimp"], O["qimpm"], f.n, f.p, f.ntree), z["local_importance"])
    assert np.array_equal(orc.finishprox(O["S"], O["nout"], full=True), z["prox"])
    err, pred, proba = orc.oob_summary(O["q_raw"], O["nout"], z["y"])
    assert np.float32(err) == z["oob_error"]
    assert np.array_equal(pred, z["oob_pred"]) and np.array_equal(proba, z["oob_proba"])
    _, tp, tpr = orc.predict(z["Xtest"], f)
    assert np.array_equal(tp, z["pred_test"]) and np.array_equal(tpr, z["proba_test"])


def test_permutations_match_golden(built):
    from oracle import oracle as orc

    z = np.load(os.path.join(GOLDEN, "permobmr.npz"))
    for k in z.files:
        noob = int(k.split("_")[1])
        perm, bad = orc.perm(noob)
        assert bad == 0
        assert np.array_equal(perm, z[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f)[:-4] for f in FILES])
def test_cuda_matches_golden(built, path):
    from rfx_b200 import abi

    z, f = load(path)
    ctx = abi.Context(0)
    ctx.load(f, z["X"], z["y"])
    q, nout, _ = ctx.route_oob()
    assert np.array_equal(q.astype(np.float32), z["q_raw"])
    assert np.array_equal(nout, z["nout"])
    err, pred, proba = ctx.oob_summary()
    assert np.float32(err) == z["oob_error"]
    assert np.array_equal(pred, z["oob_pred"]) and np.array_equal(proba, z["oob_proba"])
    S = ctx.proximity_upper()
    assert np.array_equal(ctx.finishprox(S, full=True), z["prox"])
    avimp, sqsd, qimp, qimpm = ctx.varimp(True)
    assert np.array_equal(avimp, z["importances"]) and np.array_equal(sqsd, z["sqsd"])
    assert np.array_equal(qimp, z["qimp"])
    assert np.array_equal(ctx.localimp(qimp, qimpm), z["local_importance"])
    votes = ctx.predict_votes(z["Xtest"])
    assert np.array_equal(_argmax_low(votes), z["pred_test"])
    assert np.array_equal((votes.astype(np.float32) / np.float32(f.ntree)), z["proba_test"])
    ctx.close()


def _argmax_low(votes):
    """predict_classification's vote: strict '>' so ties go to the lowest class."""
    return np.argmax(votes, axis=1).astype(np.int32)
