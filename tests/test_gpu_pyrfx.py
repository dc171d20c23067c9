"""The pybind11 mirror of the reference's rfx.RandomForestClassifier on the
GPU, against fixtures the reference's own CPU code produced (forest grown by
the reference's fit with the same configuration: maxnode = 2n + 1, mtry from
the constructor, categorical features auto-detected)."""
import os
import warnings

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
CASES = {"gauss_n300_t60": dict(mtry=3), "cover_n400_t40": dict(mtry=7)}


def procrustes_rms(A, B):
    U, _, Vt = np.linalg.svd(A.T @ B)
    R = U @ Vt
    return float(np.sqrt(np.mean((A @ R - B) ** 2))), float(np.sqrt(np.mean(B ** 2)))


def fitted(rfx, name, **kw):
    z = np.load(os.path.join(GOLD, name + ".npz"))
    n, p = z["X"].shape
    args = dict(nsample=n, ntree=int(z["nnode"].shape[0]), mdim=p, mtry=CASES[name]["mtry"], minndsize=1,
                compute_proximity=True, compute_importance=True, compute_local_importance=True, use_gpu=True,
                show_progress=False)
    args.update(kw)
    m = rfx.RandomForestClassifier(**args)
    m.fit(z["X"], z["y"])
    return z, m


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_classifier_matches_reference(built, name):
    from rfx_b200 import _rfx as rfx

    z, m = fitted(rfx, name)
    n, p = z["X"].shape
    assert m.get_n_samples() == n and m.get_n_features() == p and m.get_n_classes() == int(z["nclass"])
    assert np.float32(m.get_oob_error()) == z["oob_error"]
    oobp = m.get_oob_predictions()
    assert oobp.dtype == np.float32 and np.array_equal(oobp, z["oob_pred"].astype(np.float32))
    fi = m.feature_importances_()
    assert fi.dtype == np.float32 and np.array_equal(fi, z["importances"])
    li = m.get_local_importance()
    assert li.shape == (n, p) and np.array_equal(li, z["local_importance"])
    with pytest.warns(RuntimeWarning, match="get_proximity_matrix"):
        P = m.get_proximity_matrix()
    assert P.dtype == np.float32 and P.shape == (n, n) and np.array_equal(P, z["prox"])
    with pytest.warns(RuntimeWarning):
        P2 = m.compute_proximity_matrix()
    assert np.array_equal(P2, P)
    # held-out rows: tree votes; training-size input: the stored OOB results
    assert np.array_equal(m.predict(z["Xtest"]), z["pred_test"])
    assert np.array_equal(m.predict_proba(z["Xtest"]), z["proba_test"])
    assert np.array_equal(m.predict(z["X"]), z["oob_pred"])
    assert np.array_equal(m.predict_proba(z["X"]), z["oob_proba"])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        C = m.compute_mds_3d_cpu()
    assert C.shape == (n, 3) and C.dtype == np.float64
    rms, scale = procrustes_rms(C, z["mds3d"])
    assert rms <= 1e-6 * scale, (rms, scale)
    cm = rfx.confusion_matrix(z["y"], z["oob_pred"])
    ref = np.zeros_like(cm)
    np.add.at(ref, (z["y"], z["oob_pred"]), 1)
    assert np.array_equal(cm, ref)
    # after cleanup the forest is loaded again on demand
    m.cleanup()
    assert np.array_equal(m.predict(z["Xtest"]), z["pred_test"])
    m.cleanup()


@pytest.mark.gpu
def test_classifier_importance_flags(built):
    from rfx_b200 import _rfx as rfx

    z, m = fitted(rfx, "gauss_n300_t60", compute_proximity=False, compute_local_importance=False)
    n, p = z["X"].shape
    assert np.array_equal(m.feature_importances_(), z["importances"])
    assert not m.get_local_importance().any()
    P = m.get_proximity_matrix()  # identity when proximity was not requested
    assert np.array_equal(P, np.eye(n, dtype=np.float32))
    z, m = fitted(rfx, "gauss_n300_t60", compute_importance=False, compute_proximity=False)
    assert not m.feature_importances_().any()
    assert np.float32(m.get_oob_error()) == z["oob_error"]


@pytest.mark.gpu
@pytest.mark.parametrize("quant", ["int8", "fp32", "nf4", "fp16"])
def test_classifier_lowrank_mode(built, quant):
    from rfx_b200 import _rfx as rfx

    z, m = fitted(rfx, "cover_n400_t40", use_qlora=True, rank=16, quant_mode=quant)
    n = z["X"].shape[0]
    with pytest.raises(RuntimeError, match="Low-rank mode is active"):
        m.get_proximity_matrix()
    A, B, r = m.get_lowrank_factors()
    assert r == 16 and A.shape == (n, 16) and A.dtype == np.float64 and np.array_equal(A, B)
    F = A.ravel().reshape(r, n).T  # the column-major buffer behind the (n, r) array
    P = z["prox"].astype(np.float64)
    M = P - np.eye(n)
    err = np.linalg.norm(M - F @ F.T) / np.linalg.norm(M)
    w = np.linalg.eigvalsh(M)
    best = np.sqrt(np.sum(np.sort(np.abs(w))[:-16] ** 2)) / np.linalg.norm(M)
    # 4-bit storage adds up to half a step (1/14 of each column's maximum)
    slack = 0.08 if quant == "nf4" else 0.02
    assert err <= 1.5 * best + slack, (err, best)
    if quant == "nf4":  # every factor entry is one of the 15 code values times its column scale
        sc = np.abs(F).max(axis=0)
        codes = np.round(F / np.where(sc > 0, sc, 1) * 7)
        assert np.allclose(codes * sc / 7, F, rtol=1e-6, atol=1e-7)
    if quant == "fp16":
        assert np.array_equal(F.astype(np.float16).astype(np.float64), F)
    C = m.compute_mds_from_factors(3)
    assert C.shape == (n, 3) and C.dtype == np.float64 and np.isfinite(C).all()
    C3 = m.compute_mds_3d_from_factors()
    rms, scale = procrustes_rms(C3, C)
    assert rms <= 1e-6 * scale
    with pytest.raises(RuntimeError, match="k must be >= 1"):
        m.compute_mds_from_factors(0)
    # the other results do not depend on the proximity mode
    assert np.array_equal(m.feature_importances_(), z["importances"])
