"""Seeded synthetic datasets with the shapes of the analysis workloads.

No public dataset is read or reproduced here.  The mixed-type generator has the
*shape* of a cover-type table (10 continuous columns, one-hot groups of 4 and
40 binary columns, 7 imbalanced classes) and is otherwise invented: class
means, mixture components and one-hot probabilities are drawn from a seeded
``numpy.random.default_rng``.

Every generator returns ``(X float32 C-order (n, p), y int32 (n,))`` with
labels 0..c-1, which is the input contract of ``RandomForestClassifier.fit``
(python/randomforest_py.cpp:732).
"""
from __future__ import annotations

import numpy as np

SEED_BASE = 20251001

COVER_PRIORS = np.array([0.36, 0.49, 0.06, 0.005, 0.016, 0.03, 0.035])


def gaussian_classes(n: int = 2000, p: int = 13, c: int = 3, seed: int = SEED_BASE + 1,
                     mean_scale: float = 2.0):
    """Balanced classes, class means ~ N(0, mean_scale^2) per feature, unit noise."""
    rng = np.random.default_rng(seed)
    mu = rng.normal(0.0, mean_scale, size=(c, p))
    y = np.repeat(np.arange(c, dtype=np.int32), -(-n // c))[:n]
    # sizes 667/667/666 for n=2000, c=3: the first n % c classes get the extra row
    counts = np.full(c, n // c)
    counts[: n % c] += 1
    y = np.concatenate([np.full(k, j, dtype=np.int32) for j, k in enumerate(counts)])
    y = rng.permutation(y).astype(np.int32)
    X = mu[y] + rng.normal(size=(n, p))
    return np.ascontiguousarray(X, dtype=np.float32), y


def mixed_cover(n: int = 50_000, seed: int = SEED_BASE + 2, mean_scale: float = 1.0,
                t_frac: float = 0.05):
    """p = 54: 10 continuous + one-hot(4) + one-hot(40); 7 imbalanced classes.

    Continuous columns: per class a two-component Gaussian mixture with shifted
    means; a fraction ``t_frac`` of the noise entries is Student-t(3).
    Binary columns: each group is one-hot with class-dependent Dirichlet
    probabilities.  Binary columns hold exactly 0.0/1.0, so the categorical
    auto-detection of ``fit`` marks them as 2-level categoricals.
    """
    rng = np.random.default_rng(seed)
    c = len(COVER_PRIORS)
    y = rng.choice(c, size=n, p=COVER_PRIORS / COVER_PRIORS.sum()).astype(np.int32)
    # make sure every class occurs (nclass is counted from the labels)
    for j in range(c):
        if not np.any(y == j):
            y[rng.integers(n)] = j
    mu = rng.normal(0.0, mean_scale, size=(c, 2, 10))
    comp = rng.integers(0, 2, size=n)
    noise = rng.normal(size=(n, 10))
    heavy = rng.random(size=(n, 10)) < t_frac
    noise[heavy] = rng.standard_t(3, size=int(heavy.sum()))
    cont = mu[y, comp] + noise
    X = np.zeros((n, 54), dtype=np.float32)
    X[:, :10] = cont
    for start, width, alpha in ((10, 4, 1.0), (14, 40, 0.3)):
        probs = rng.dirichlet(np.full(width, alpha), size=c)
        # sample one category per row from its class's distribution
        u = rng.random(n)
        cdf = np.cumsum(probs, axis=1)
        cdf[:, -1] = 1.0
        k = (u[:, None] > cdf[y]).sum(axis=1)
        X[np.arange(n), start + k] = 1.0
    return np.ascontiguousarray(X), y


def uneven_forests(count: int = 64, seed: int = SEED_BASE + 4, n_range=(1000, 50_000),
                   p_range=(8, 100), c_range=(2, 10)):
    """Specs of many independent forests of uneven size: list of dicts with X, y, mtry."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        p = int(rng.integers(p_range[0], p_range[1] + 1))
        c = int(rng.integers(c_range[0], c_range[1] + 1))
        n_noise = int(round(0.3 * p))
        y = rng.integers(0, c, size=n).astype(np.int32)
        for j in range(c):
            if not np.any(y == j):
                y[rng.integers(n)] = j
        mu = rng.normal(0.0, 1.5, size=(c, p - n_noise))
        X = np.empty((n, p), dtype=np.float32)
        X[:, : p - n_noise] = mu[y] + rng.normal(size=(n, p - n_noise))
        X[:, p - n_noise:] = rng.normal(size=(n, n_noise))
        out.append({"X": np.ascontiguousarray(X), "y": y, "mtry": int(np.floor(np.sqrt(p)))})
    return out


def large_gmm(n: int = 1_000_000, p: int = 32, seed: int = SEED_BASE + 5, n_comp: int = 8,
              n_class: int = 4, outlier_frac: float = 0.01, return_outliers: bool = False):
    """8-component Gaussian mixture, 4 classes, 1% uniform outliers in a 10x box
    (with return_outliers, also the sorted indices of the injected outliers)."""
    rng = np.random.default_rng(seed)
    centers = rng.normal(0.0, 3.0, size=(n_comp, p))
    comp_class = np.arange(n_comp) % n_class
    comp = rng.integers(0, n_comp, size=n)
    X = centers[comp] + rng.normal(size=(n, p))
    y = comp_class[comp].astype(np.int32)
    n_out = int(round(outlier_frac * n))
    idx = rng.choice(n, size=n_out, replace=False)
    lo, hi = X.min(axis=0), X.max(axis=0)
    mid, half = 0.5 * (lo + hi), 0.5 * (hi - lo)
    X[idx] = mid + rng.uniform(-10.0, 10.0, size=(n_out, p)) * half
    y[idx] = rng.integers(0, n_class, size=n_out)
    if return_outliers:
        return np.ascontiguousarray(X, dtype=np.float32), y, np.sort(idx)
    return np.ascontiguousarray(X, dtype=np.float32), y


def detect_categorical(X: np.ndarray, maxcat: int = 10) -> np.ndarray:
    """Categorical auto-detection of ``fit`` (python/randomforest_py.cpp:773-803).

    A column is categorical, with ``cat[m]`` = its number of distinct values,
    when every value is within 1e-5 of an integer, it has 2..maxcat distinct
    values, and all values lie in [0, maxcat).  Other columns get ``cat[m] = 1``.
    """
    X = np.asarray(X, dtype=np.float32)
    n, p = X.shape
    cat = np.ones(p, dtype=np.int32)
    for m in range(p):
        col = X[:, m]
        # std::round rounds half away from zero; np.round rounds half to even.
        r = np.where(col >= 0, np.floor(col + np.float32(0.5)), np.ceil(col - np.float32(0.5)))
        if np.any(np.abs(col - r.astype(np.float32)) > np.float32(1e-5)):
            continue
        u = np.unique(col)
        if 1 < u.size <= maxcat and col.min() >= 0.0 and col.max() < np.float32(maxcat):
            cat[m] = u.size
    return cat
