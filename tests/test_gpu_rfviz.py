"""The rfviz data feed (rfx_b200.rfviz.rfviz_data) from the drop-in
classifier on the plain-method configuration (n=2000, p=13, 3 classes,
500 trees): the arrays the reference's dashboard plots, compared with the same
derivation applied to the reference's own outputs (tests/golden/
config1_n2000_t500.npz): local importance and its normalisation, OOB
predictions and the one-hot vote matrix bit for bit, the proximity matrix by
digest, the 3-D MDS within a Procrustes RMS of 1e-6 x scale, and the KMeans
partition (k-means++ and Lloyd steps depend on distances only, so a rotated
embedding gives the same clusters)."""
import os
import warnings

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _same_partition(a, b):
    pairs = set(zip(a.tolist(), b.tolist()))
    return len(pairs) == len(set(a.tolist())) == len(set(b.tolist()))


def test_rfviz_feed_matches_reference_outputs(built):
    from sklearn.cluster import KMeans

    from rfx_b200 import _rfx as rfx
    from rfx_b200.rfviz import rfviz_data
    from test_config_parity import _check_prox, _procrustes

    z = np.load(os.path.join(ROOT, "tests", "golden", "config1_n2000_t500.npz"))
    n, p = z["X"].shape
    m = rfx.RandomForestClassifier(nsample=n, ntree=int(z["ntree"]), mdim=p, mtry=int(z["mtry"]), minndsize=1,
                                   compute_proximity=True, compute_importance=True, compute_local_importance=True,
                                   use_gpu=True, show_progress=False)
    m.fit(z["X"], z["y"])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        d = rfviz_data(m, z["X"], z["y"], n_clusters=3)
    li = z["local_importance"]
    assert np.array_equal(d["local_imp"], li)
    ref_norm = (li - li.min(axis=0, keepdims=True)) / (li.max(axis=0, keepdims=True) - li.min(axis=0, keepdims=True)
                                                       + 1e-10)
    assert np.array_equal(d["local_imp_normalized"], ref_norm)
    assert np.array_equal(d["oob_pred"], z["oob_pred"].astype(int))
    assert np.array_equal(d["vote_matrix"].argmax(axis=1), z["oob_pred"]) and d["vote_matrix"].sum() == n
    _check_prox(d["proximity"], z)
    rms, scale = _procrustes(d["coords_3d"], z["mds3d"])
    assert rms <= 1e-6 * scale
    assert d["valid_mask"].all() and d["extra_dims"] is None
    ref_labels = KMeans(n_clusters=3, random_state=42, n_init=10).fit_predict(z["mds3d"])
    assert _same_partition(d["cluster_labels"], ref_labels)
    assert d["feature_names"] == [f"Feature {i}" for i in range(p)]
    # the elbow rule when no cluster count is given
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        d2 = rfviz_data(m, z["X"], z["y"], n_clusters=None)
    assert 3 <= d2["n_clusters"] <= 9
    m.cleanup()
