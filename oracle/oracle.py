"""ctypes front-end of the oracle (oracle/oracle.c) — test infrastructure only.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
checker; the product path never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build() -> None:
    subprocess.run(["make", "-s", "-f", os.path.join(HERE, "Makefile"), "oracle"], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = ctypes.CDLL(path)
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def perm(noob: int):
    """(perm, bad): cpu_permobmr's permutation of OOB positions for this noob."""
    out = np.empty(max(noob, 1), dtype=np.int32)
    bad = lib().orc_perm(ctypes.c_int(noob), _p(out))
    return out[:noob], int(bad)


def bootstrap(n: int, tree: int) -> np.ndarray:
    nin = np.empty(n, dtype=np.int32)
    lib().orc_bootstrap(ctypes.c_int(n), ctypes.c_int(tree), _p(nin))
    return nin


def analyse(X, y, forest, do_imp=True, impn=True, do_prox=True, want_leaf=False, want_jtr=False, S=None,
            casewise=False, want_cw=False):
    """Whole-forest analysis in the reference's per-tree order (see orc_analyse).

    With ``S`` (int32, n(n+1)/2, C-contiguous) the pair counts are added to
    that buffer instead of a fresh zeroed one, as the reference accumulates
    one proximity array over all trees.  ``casewise`` weights votes,
    importance and the FP64 proximity sums as the reference's
    use_casewise=True; ``want_cw`` returns those FP64 sums as ``Cw`` (n x n,
    row = OOB sample, column = in-bag sample) and their packed symmetric
    upper triangle ``Sd`` = C + C^T."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.int32)
    f = forest
    n, p, c, T = f.n, f.p, f.nclass, f.ntree
    out = dict(
        q_raw=np.zeros(n * c, np.float32), nout=np.zeros(n, np.int32),
        qimp=np.zeros(n, np.float32), qimpm=np.zeros(n * p, np.float32),
        avimp=np.zeros(p, np.float32), sqsd=np.zeros(p, np.float32))
    if not do_prox:
        S = None
    elif S is None:
        S = np.zeros(n * (n + 1) // 2, np.int32)
    elif S.dtype != np.int32 or S.size != n * (n + 1) // 2 or not S.flags.c_contiguous:
        raise ValueError("S must be a C-contiguous int32 array of n(n+1)/2 entries")
    Cw = np.zeros(n * n, np.float64) if want_cw else None
    leaf = np.zeros(T * n, np.int32) if want_leaf else None
    jtr = np.zeros(T * n, np.int32) if want_jtr else None
    bad = ctypes.c_int(0)
    offs = np.ascontiguousarray(f.offs[:-1], dtype=np.int64)
    lib().orc_analyse(
        _p(X), _p(y), _p(f.cat), n, p, c, f.maxcat, T, _p(offs), _p(f.nnode), _p(f.nodestatus),
        _p(f.bestvar), _p(f.xbestsplit), _p(f.treemap), _p(f.nodeclass), _p(f.catgoleft), _p(f.nin),
        int(bool(do_imp)), int(bool(impn)), int(bool(do_prox)), int(bool(casewise)),
        _p(out["q_raw"]), _p(out["nout"]), _p(out["qimp"]), _p(out["qimpm"]), _p(out["avimp"]),
        _p(out["sqsd"]), _p(S), _p(Cw), _p(leaf), _p(jtr), ctypes.byref(bad))
    out["q_raw"] = out["q_raw"].reshape(n, c)
    out["S"] = S
    if want_cw:
        C = Cw.reshape(n, n)
        iu = np.triu_indices(n)
        out["Cw"] = C
        out["Sd"] = np.ascontiguousarray((C + C.T)[iu])
    out["leaf"] = None if leaf is None else leaf.reshape(T, n)
    out["jtr"] = None if jtr is None else jtr.reshape(T, n)
    out["perm_bad"] = int(bad.value)
    return out


def pairs_from_leaves(leaf, inbag, max_leaves):
    """Pair counts (packed upper triangle, int32) from per-(tree, sample)
    terminal indices and bag flags: cpu_proximity's dense branch without the
    routing (see orc_pairs_from_leaves).  Returns (S, number of indices
    >= max_leaves that were left out)."""
    leaf = np.ascontiguousarray(leaf, dtype=np.int32)
    inbag = np.ascontiguousarray(inbag != 0, dtype=np.uint8)
    T, n = leaf.shape
    S = np.zeros(n * (n + 1) // 2, np.int32)
    f = lib().orc_pairs_from_leaves
    f.restype = ctypes.c_int64
    bad = f(ctypes.c_int(n), ctypes.c_int(T), ctypes.c_int(max_leaves), _p(leaf), _p(inbag), _p(S))
    return S, int(bad)


def oob_summary(q_raw, nout, y):
    n, c = q_raw.shape
    err = ctypes.c_float(0)
    pred = np.zeros(n, np.int32)
    proba = np.zeros((n, c), np.float32)
    lib().orc_oob_summary(n, c, _p(np.ascontiguousarray(q_raw, np.float32)), _p(np.ascontiguousarray(nout, np.int32)),
                          _p(np.ascontiguousarray(y, np.int32)), ctypes.byref(err), _p(pred), _p(proba))
    return float(err.value), pred, proba


def finishprox(S, nout, full=True, double=False):
    n = nout.size
    size = n * n if full else n * (n + 1) // 2
    P = None if double else np.zeros(size, np.float32)
    Pd = np.zeros(size, np.float64) if double else None
    lib().orc_finishprox(n, _p(np.ascontiguousarray(S, np.int32)), _p(np.ascontiguousarray(nout, np.int32)),
                         int(bool(full)), _p(P), _p(Pd))
    R = Pd if double else P
    return R.reshape(n, n) if full else R


def finishprox_f64(Sd, nout, full=True):
    """orc_finishprox_f64: cpu_finishprox from the packed FP64 sums C + C^T."""
    n = nout.size
    P = np.zeros(n * n if full else n * (n + 1) // 2, np.float32)
    lib().orc_finishprox_f64(n, _p(np.ascontiguousarray(Sd, np.float64)), _p(np.ascontiguousarray(nout, np.int32)),
                             int(bool(full)), _p(P), None)
    return P.reshape(n, n) if full else P


def rfgap(nin, node):
    """orc_rfgap: the RF-GAP proximity matrix (n x n FP64) from per-tree
    multiplicities and node ids (T x n each)."""
    nin = np.ascontiguousarray(nin, np.int32)
    node = np.ascontiguousarray(node, np.int32)
    T, n = nin.shape
    P = np.zeros(n * n, np.float64)
    lib().orc_rfgap(n, T, _p(nin), _p(node), _p(P))
    return P.reshape(n, n)


def localimp(qimp, qimpm, n, p, T):
    out = np.zeros(n * p, np.float32)
    lib().orc_localimp(n, p, T, _p(np.ascontiguousarray(qimp, np.float32)),
                       _p(np.ascontiguousarray(qimpm, np.float32)), _p(out))
    return out.reshape(n, p)


def predict(Xt, forest):
    Xt = np.ascontiguousarray(Xt, dtype=np.float32)
    f = forest
    m = Xt.shape[0]
    votes = np.zeros(m * f.nclass, np.int32)
    pred = np.zeros(m, np.int32)
    proba = np.zeros(m * f.nclass, np.float32)
    offs = np.ascontiguousarray(f.offs[:-1], dtype=np.int64)
    lib().orc_predict(_p(Xt), m, f.p, f.nclass, f.maxcat, f.n, f.ntree, _p(offs), _p(f.nnode), _p(f.nodestatus),
                      _p(f.bestvar), _p(f.xbestsplit), _p(f.treemap), _p(f.nodeclass), _p(f.catgoleft),
                      _p(f.cat), _p(votes), _p(pred), _p(proba))
    return votes.reshape(m, f.nclass), pred, proba.reshape(m, f.nclass)


def upper_to_full(S_upper, n):
    """Expand a packed row-major upper triangle (diagonal included) to n x n."""
    M = np.zeros((n, n), dtype=S_upper.dtype)
    iu = np.triu_indices(n)
    M[iu] = S_upper
    M.T[iu] = S_upper
    return M
