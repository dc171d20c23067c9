"""ctypes front-end of oracle/_ref/librfxref.so — the reference's own CPU code.

Test infrastructure only (tests/, smoke(), bench.py's reference arm).  The
library is built by ``make -f oracle/Makefile REF_DIR=<reference checkout> ref`` from the reference's
sources where they lie; it is absent when the reference tree was not available
at build time, in which case ``available()`` is False.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from rfx_b200.forest import Forest

HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(HERE, "_ref", "librfxref.so")
_LIB = None


def available() -> bool:
    return os.path.exists(PATH)


def lib():
    global _LIB
    if _LIB is None:
        _LIB = ctypes.CDLL(PATH)
        _LIB.rh_last_error.restype = ctypes.c_char_p
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().rh_last_error().decode())


def set_threads(n: int) -> int:
    return int(lib().rh_set_threads(int(n)))


def fit_capture(X, y, cat, ntree, mtry=0, minndsize=1, maxcat=10, iseed=12345,
                compute_proximity=True, compute_importance=True, compute_local_importance=True,
                use_casewise=False, use_rfgap=False):
    """Run rf::RandomForest::fit on the CPU path and capture everything."""
    X = np.ascontiguousarray(X, np.float32)
    y = np.ascontiguousarray(y, np.int32)
    cat = np.ascontiguousarray(cat, np.int32)
    n, p = X.shape
    T = ntree
    mx = 2 * n + 1
    c_guess = int(np.unique(y).size)
    a = dict(
        nnode=np.zeros(T, np.int32), nodestatus=np.zeros(T * mx, np.int32), bestvar=np.zeros(T * mx, np.int32),
        xbestsplit=np.zeros(T * mx, np.float32), treemap=np.zeros(T * 2 * mx, np.int32),
        nodeclass=np.zeros(T * mx, np.int32), nin=np.zeros(T * n, np.int32), jtr=np.zeros(T * n, np.int32),
        nodextr=np.zeros(T * n, np.int32), q_raw=np.zeros(n * c_guess, np.float32), nout=np.zeros(n, np.int32),
        scalars=np.zeros(4, np.float32), oob_pred=np.zeros(n, np.int32), oob_proba=np.zeros(n * c_guess, np.float32),
        importances=np.zeros(p, np.float32), qimp=np.zeros(n, np.float32), qimpm=np.zeros(n * p, np.float32),
        avimp=np.zeros(p, np.float32), sqsd=np.zeros(p, np.float32))
    prox = np.zeros(n * n, np.float64) if compute_proximity else None
    nclass = ctypes.c_int(0)
    _check(lib().rh_fit_capture(
        _p(X), _p(y), _p(cat), n, p, T, mtry, minndsize, maxcat, iseed,
        int(compute_proximity), int(compute_importance), int(compute_local_importance), int(use_casewise),
        int(use_rfgap), ctypes.byref(nclass),
        *[_p(a[k]) for k in ("nnode", "nodestatus", "bestvar", "xbestsplit", "treemap", "nodeclass", "nin", "jtr",
                             "nodextr", "q_raw", "nout", "scalars", "oob_pred", "oob_proba", "importances", "qimp",
                             "qimpm", "avimp", "sqsd")], _p(prox)))
    c = nclass.value
    forest = Forest.from_padded(n, p, c, maxcat, a["nnode"], a["nodestatus"], a["bestvar"], a["xbestsplit"],
                                a["treemap"], a["nodeclass"], a["nin"], cat)
    return dict(
        forest=forest, nclass=c, jtr=a["jtr"].reshape(T, n), nodextr=a["nodextr"].reshape(T, n),
        q_raw=a["q_raw"].reshape(n, c), nout=a["nout"], oob_error=float(a["scalars"][0]), oob_pred=a["oob_pred"],
        oob_proba=a["oob_proba"].reshape(n, c), importances=a["importances"], qimp=a["qimp"],
        qimpm=a["qimpm"].reshape(n, p), avimp=a["avimp"], sqsd=a["sqsd"],
        prox=None if prox is None else prox.reshape(n, n).T.copy())  # column-major -> [row][col]


def grow_forest(X, y, ntree, mtry, minndsize=1, maxcat=10, iseed=12345, cat=None) -> Forest:
    """cpu_bootstrap + cpu_growtree_wrapper per tree (parallel over trees)."""
    X = np.ascontiguousarray(X, np.float32)
    y = np.ascontiguousarray(y, np.int32)
    n, p = X.shape
    c = int(y.max()) + 1
    T = ntree
    mx = 2 * n + 1
    nnode = np.zeros(T, np.int32)
    ns = np.zeros(T * mx, np.int32)
    bv = np.zeros(T * mx, np.int32)
    xs = np.zeros(T * mx, np.float32)
    tm = np.zeros(T * 2 * mx, np.int32)
    nc = np.zeros(T * mx, np.int32)
    nin = np.zeros(T * n, np.int32)
    _check(lib().rh_grow_forest(_p(X), _p(y), n, p, c, T, mtry, minndsize, maxcat, iseed, _p(nnode), _p(ns), _p(bv),
                                _p(xs), _p(tm), _p(nc), _p(nin)))
    if cat is None:
        cat = np.ones(p, np.int32)
    return Forest.from_padded(n, p, c, maxcat, nnode, ns, bv, xs, tm, nc, nin, cat)


def analyse_trees(X, y, forest, t0=0, t1=None, do_imp=True, impn=True, do_prox=False, want_leaf=False, state=None):
    """The per-tree analysis sequence of grow_tree_single for trees [t0, t1).

    ``state`` carries the accumulators (q, nout, qimp, qimpm, avimp, sqsd,
    prox) between calls so a forest can be analysed in slices."""
    X = np.ascontiguousarray(X, np.float32)
    y = np.ascontiguousarray(y, np.int32)
    f = forest
    n, p, c = f.n, f.p, f.nclass
    t1 = f.ntree if t1 is None else t1
    if state is None:
        state = dict(q=np.zeros(n * c, np.float32), nout=np.zeros(n, np.int32), qimp=np.zeros(n, np.float32),
                     qimpm=np.zeros(n * p, np.float32), avimp=np.zeros(p, np.float32), sqsd=np.zeros(p, np.float32),
                     prox=np.zeros(n * n, np.float64) if do_prox else None)
    leaf = np.zeros((t1 - t0) * n, np.int32) if want_leaf else None
    offs = np.ascontiguousarray(f.offs[:-1], dtype=np.int64)
    _check(lib().rh_analyse_trees(
        _p(X), _p(y), _p(f.cat), n, p, c, f.maxcat, t0, t1, _p(offs), _p(f.nnode), _p(f.nodestatus), _p(f.bestvar),
        _p(f.xbestsplit), _p(f.treemap), _p(f.nodeclass), _p(f.catgoleft), _p(f.nin), int(do_imp), int(impn),
        _p(state["q"]), _p(state["nout"]), _p(state["qimp"]), _p(state["qimpm"]), _p(state["avimp"]),
        _p(state["sqsd"]), _p(state["prox"]), _p(leaf)))
    if want_leaf:
        state["leaf"] = leaf.reshape(t1 - t0, n)
    return state


def permobmr(noob: int) -> np.ndarray:
    """The reference's cpu_permobmr permutation of OOB positions 0..noob-1."""
    out = np.zeros(max(noob, 1), np.int32)
    lib().rh_permobmr(int(noob), _p(out))
    return out[:noob]


def finishprox(prox_rowmajor, nout):
    """cpu_finishprox on a square [row][col] matrix; returns [row][col]."""
    n = nout.size
    colmajor = np.ascontiguousarray(np.asarray(prox_rowmajor, np.float64).T)
    out = np.zeros_like(colmajor)
    lib().rh_finishprox(n, _p(np.ascontiguousarray(nout, np.int32)), _p(colmajor), _p(out))
    return out.T.copy()


def localimp(qimp, qimpm, n, p, T):
    q = np.ascontiguousarray(qimpm, np.float32).reshape(-1).copy()
    lib().rh_localimp(n, p, T, _p(np.ascontiguousarray(qimp, np.float32)), _p(q))
    return q.reshape(n, p)


def mds3d(P_float32, nout):
    """compute_mds_3d_cpu as the binding calls it: float32 P promoted to FP64."""
    n = nout.size
    Pd = np.ascontiguousarray(np.asarray(P_float32, np.float32).astype(np.float64))
    coords = np.zeros(n * 3, np.float64)
    _check(lib().rh_mds3d(_p(Pd), n, _p(np.ascontiguousarray(nout, np.int32)), _p(coords)))
    return coords.reshape(n, 3)


def predict(Xt, forest):
    Xt = np.ascontiguousarray(Xt, np.float32)
    f = forest
    n, T = f.n, f.ntree
    mx = 2 * n + 1
    pad = lambda a, k=1: np.concatenate([np.pad(a[k * f.offs[t]: k * f.offs[t + 1]], (0, k * (mx - f.nnode[t])))
                                         for t in range(T)])
    m = Xt.shape[0]
    pred = np.zeros(m, np.int32)
    proba = np.zeros(m * f.nclass, np.float32)
    _check(lib().rh_predict(n, f.p, f.nclass, T, f.maxcat, _p(f.cat), _p(f.nnode), _p(pad(f.nodestatus)),
                            _p(pad(f.bestvar)), _p(pad(f.xbestsplit)), _p(pad(f.treemap, 2)), _p(pad(f.nodeclass)),
                            _p(None if f.catgoleft is None else pad(f.catgoleft, f.maxcat)),
                            _p(Xt), m, _p(pred), _p(proba)))
    return pred, proba.reshape(m, f.nclass)
