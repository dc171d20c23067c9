"""The data feed of the reference's ``rfx.rfviz`` dashboard.

``rfx.rfviz`` (python/randomforest_py.cpp:2821-4137) takes a fitted model and
builds a 2 x 2 plotly figure: parallel coordinates of the input features and
of the normalised local importance, a 3-D MDS scatter coloured by KMeans
cluster, and a heat map of OOB class votes.  Everything it plots comes from
the model's analysis path (local importance, OOB predictions, proximity or
its low-rank factors, MDS coordinates), which this library computes on the
GPU.  :func:`rfviz_data` returns those arrays, derived exactly as the
reference's embedded Python derives them (the same getters in the same
fallback order, the same normalisations, the same elbow rule for the cluster
count, KMeans with random_state=42 and n_init=10), so that the reference's
HTML generator, or any other front end, can be fed from this library.

The HTML/WebGL rendering itself (plotly traces, the injected JavaScript for
linked brushing) is not part of the analysis path and is not reproduced.
"""
from __future__ import annotations

from typing import Optional

import numpy as np


def _coords(rf_model, mds_k: int):
    """MDS coordinates in the reference's order: compute_mds_from_factors(k)
    (low-rank mode), else compute_mds_3d_cpu() for k == 3
    (python/randomforest_py.cpp:2956-2988)."""
    gpu_err = None
    coords = None
    try:
        c = rf_model.compute_mds_from_factors(k=mds_k)
        if c is not None:
            coords = np.asarray(c)
    except Exception as e:  # low-rank factors not available
        gpu_err = str(e)
    if coords is None:
        if mds_k != 3:
            raise RuntimeError(f"Cannot compute MDS: GPU low-rank MDS failed ({gpu_err}) and CPU MDS only supports "
                               f"k=3 (requested k={mds_k}).")
        try:
            coords = np.asarray(rf_model.compute_mds_3d_cpu())
        except Exception as e2:
            raise RuntimeError(f"Cannot compute MDS: GPU low-rank MDS failed ({gpu_err or 'unknown error'}) and CPU "
                               f"MDS failed ({e2}).")
    return coords


def _to_3d(coords_kd: np.ndarray):
    """First three MDS dimensions (padded with zeros below three) and the
    extra ones (python/randomforest_py.cpp:2990-3007)."""
    n = coords_kd.shape[0]
    k = coords_kd.shape[1]
    if k >= 3:
        return coords_kd[:, :3], (coords_kd[:, 3:] if k > 3 else None)
    if k == 2:
        return np.column_stack([coords_kd, np.zeros(n)]), None
    if k == 1:
        return np.column_stack([coords_kd, np.zeros(n), np.zeros(n)]), None
    raise RuntimeError(f"Invalid MDS dimensions: {k}")


def _elbow(coords_3d, n_classes: int, n_samples: int) -> int:
    """Cluster count by the reference's WCSS percentage-decrease rule
    (threshold 5 %, python/randomforest_py.cpp:3016-3049)."""
    from sklearn.cluster import KMeans

    max_k = min(15, n_samples // 10, n_classes * 3)
    min_k = max(2, n_classes)
    if max_k < min_k:
        return min_k
    ks = list(range(min_k, max_k + 1))
    wcss = []
    for k in ks:
        km = KMeans(n_clusters=k, random_state=42, n_init=10, max_iter=300)
        km.fit(coords_3d)
        wcss.append(km.inertia_)
    optimal = min_k
    for i in range(1, len(wcss)):
        if wcss[i - 1] > 0:
            if (wcss[i - 1] - wcss[i]) / wcss[i - 1] * 100.0 < 5.0:
                optimal = ks[i - 1]
                break
        optimal = ks[i]
    return optimal


def _scale(v, lo_out: float, span: float, const: float):
    mn, mx = v.min(), v.max()
    if mx > mn:
        return lo_out + span * (v - mn) / (mx - mn)
    return np.ones(v.shape[0]) * const


def rfviz_data(rf_model, X, y, feature_names=None, n_clusters: Optional[int] = 3, mds_k: int = 3) -> dict:
    """Every array the reference's rfviz plots, from a fitted model.

    Keys: ``local_imp`` (n, p) and ``local_imp_normalized`` (column-wise
    min-max with the reference's 1e-10 guard), ``proximity`` (n, n float32 or
    None in low-rank mode), ``oob_pred`` (int), ``vote_matrix`` (n, classes,
    one-hot of the OOB prediction), ``coords_kd`` / ``coords_3d`` /
    ``extra_dims`` (MDS), ``valid_mask`` (finite coordinates), ``n_clusters``
    (given, or by the elbow rule when None or <= 0), ``cluster_labels``
    (KMeans on coords_3d), ``dim4_color`` / ``dim5_size`` / ``dim6_opacity``
    (extra MDS dimensions as visual channels, or None), ``feature_names``,
    ``unique_classes`` and ``colors`` (label -> hsl string)."""
    import warnings

    from sklearn.cluster import KMeans

    X = np.asarray(X)
    y = np.asarray(y)
    local_imp = np.asarray(rf_model.get_local_importance())
    proximity = None
    try:
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            proximity = rf_model.get_proximity_matrix()
    except Exception:
        proximity = None
    try:
        oob_pred = np.asarray(rf_model.get_oob_predictions()).astype(int)
    except Exception:
        oob_pred = np.asarray(rf_model.predict(X)).astype(int)
    if feature_names is None:
        feature_names = [f"Feature {i}" for i in range(X.shape[1])]
    norm = (local_imp - np.min(local_imp, axis=0, keepdims=True)) / (
        np.max(local_imp, axis=0, keepdims=True) - np.min(local_imp, axis=0, keepdims=True) + 1e-10)
    unique_classes = np.unique(y)
    n_classes = len(unique_classes)
    n_samples = X.shape[0]
    vote_matrix = np.zeros((n_samples, n_classes))
    vote_matrix[np.arange(n_samples), oob_pred] = 1.0
    colors = {label: f"hsl({i * 360 // len(unique_classes)}, 70%, 50%)" for i, label in enumerate(unique_classes)}
    coords_kd = _coords(rf_model, mds_k)
    coords_3d, extra = _to_3d(coords_kd)
    valid_mask = np.all(np.isfinite(coords_3d), axis=1)
    if n_clusters is None or n_clusters <= 0:
        n_clusters = _elbow(coords_3d, n_classes, n_samples)
    dim4 = dim5 = dim6 = None
    if extra is not None and extra.shape[1] > 0:
        dim4 = _scale(extra[:, 0], 0.0, 1.0, 0.5)
        if extra.shape[1] >= 2:
            dim5 = _scale(extra[:, 1], 3.0, 7.0, 6.5)
        if extra.shape[1] >= 3:
            dim6 = _scale(extra[:, 2], 0.3, 0.7, 0.65)
    labels = KMeans(n_clusters=n_clusters, random_state=42, n_init=10).fit_predict(coords_3d)
    return dict(local_imp=local_imp, local_imp_normalized=norm, proximity=proximity, oob_pred=oob_pred,
                vote_matrix=vote_matrix, coords_kd=coords_kd, coords_3d=coords_3d, extra_dims=extra,
                valid_mask=valid_mask, n_clusters=int(n_clusters), cluster_labels=labels, dim4_color=dim4,
                dim5_size=dim5, dim6_opacity=dim6, feature_names=list(feature_names),
                unique_classes=unique_classes, colors=colors)
