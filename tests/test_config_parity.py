"""Parity at the configurations the benchmark and the reference's own CPU path
are quoted on, not only at small cases.

* config1_n2000_t500 — the plain method at its stated shape (n=2000, p=13,
  3 balanced Gaussian classes, ntree=500, mtry=3, nodesize 1).  The golden
  fixture was written by tests/golden/make_golden.py from the reference's own
  fit, compute_mds_3d_cpu and predict (oracle/_ref).  Checked: the library's
  grower reproduces the reference's forest bit for bit (SHA-256); the oracle
  (CPU) and the CUDA path through the C ABI and through the pybind11 mirror
  reproduce the OOB votes, nout, error, predictions, probabilities,
  importances, local importance, the float32 proximity matrix (SHA-256 of its
  bytes, row sums, complete rows) and test-set predictions bit for bit; the
  full-matrix 3-D MDS within a Procrustes RMS of 1e-6 x scale.
* the benchmarked exact workload — n=50,000, p=54 mixed-type cover-shaped
  rows, the bench's own forest (same generator, seed, mtry 7, nodesize 1,
  1000 trees), of which 200 trees are analysed: the 20 trees with the most
  pair updates plus 180 others in seeded random order.  The CUDA path is
  compared with the oracle (oracle/oracle.c) on the same trees: leaf ids of
  every (tree, sample), OOB votes, nout, all four importance arrays and the
  local importance in full, the whole INT32 upper-triangle S (1.25e9
  entries), and finishprox on 2,000 rows (the members of the largest hub
  leaves among them) against the oracle's finishprox of the same S.
"""
import hashlib
import os
import sys
import warnings

import numpy as np
import pytest

from conftest import ROOT
from rfx_b200.forest import Forest

GOLDEN = os.path.join(ROOT, "tests", "golden")
C1 = os.path.join(GOLDEN, "config1_n2000_t500.npz")
FOREST_FIELDS = ("nnode", "nodestatus", "bestvar", "xbestsplit", "treemap", "nodeclass", "nin")


def _digest(a) -> str:
    a = np.ascontiguousarray(a)
    return hashlib.sha256(str(a.dtype).encode() + str(a.shape).encode() + a.tobytes()).hexdigest()


def _forest_digest(f) -> str:
    h = hashlib.sha256()
    for k in FOREST_FIELDS:
        a = np.ascontiguousarray(getattr(f, k))
        h.update(k.encode())
        h.update(str(a.dtype).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def _config1():
    z = np.load(C1)
    n, p = z["X"].shape
    nnode = z["nnode"]
    offs = np.zeros(nnode.size + 1, np.int64)
    offs[1:] = np.cumsum(nnode)
    f = Forest(n, p, int(z["nclass"]), int(z["maxcat"]), nnode, offs, z["nodestatus"], z["bestvar"],
               z["xbestsplit"], z["treemap"], z["nodeclass"], z["nin"].reshape(-1, n), z["cat"])
    return z, f


def _check_prox(P, z):
    assert P.dtype == np.float32 and P.shape == (2000, 2000)
    assert np.array_equal(P[z["prox_rows_idx"]], z["prox_rows"])
    assert np.array_equal(P.astype(np.float64).sum(axis=1), z["prox_rowsum"])
    assert _digest(P) == str(z["prox_sha256"])


def _procrustes(C, R):
    U, _, Vt = np.linalg.svd(C.T @ R)
    return float(np.sqrt(np.mean((C @ (U @ Vt) - R) ** 2))), float(np.sqrt(np.mean(R ** 2)))


def test_config1_forest_is_the_reference_forest(built):
    """The stored forest is the one the reference grew (digest), and the
    library's grower, which `fit` uses, reproduces it bit for bit."""
    from rfx_b200 import abi

    z, f = _config1()
    assert _forest_digest(f) == str(z["forest_sha256"])
    g = abi.grow_forest(z["X"], z["y"], int(z["ntree"]), int(z["mtry"]), int(z["minndsize"]),
                        nclass=int(z["nclass"]), cat=z["cat"])
    assert _forest_digest(g) == str(z["forest_sha256"])


def test_config1_oracle_matches_reference(built):
    from oracle import oracle as orc

    z, f = _config1()
    O = orc.analyse(z["X"], z["y"], f)
    assert np.array_equal(O["q_raw"], z["q_raw"]) and np.array_equal(O["nout"], z["nout"])
    assert np.array_equal(O["avimp"], z["importances"]) and np.array_equal(O["sqsd"], z["sqsd"])
    assert np.array_equal(O["qimp"], z["qimp"])
    assert np.array_equal(orc.localimp(O["qimp"], O["qimpm"], f.n, f.p, f.ntree), z["local_importance"])
    _check_prox(orc.finishprox(O["S"], O["nout"], full=True), z)
    err, pred, proba = orc.oob_summary(O["q_raw"], O["nout"], z["y"])
    assert np.float32(err) == z["oob_error"]
    assert np.array_equal(pred, z["oob_pred"]) and np.array_equal(proba, z["oob_proba"])
    _, tp, tpr = orc.predict(z["Xtest"], f)
    assert np.array_equal(tp, z["pred_test"]) and np.array_equal(tpr, z["proba_test"])


@pytest.mark.gpu
def test_config1_cuda_matches_reference(built):
    from rfx_b200 import abi

    z, f = _config1()
    ctx = abi.Context(0)
    ctx.load(f, z["X"], z["y"])
    q, nout, _ = ctx.route_oob()
    assert np.array_equal(q.astype(np.float32), z["q_raw"]) and np.array_equal(nout, z["nout"])
    err, pred, proba = ctx.oob_summary()
    assert np.float32(err) == z["oob_error"]
    assert np.array_equal(pred, z["oob_pred"]) and np.array_equal(proba, z["oob_proba"])
    P = ctx.finishprox(ctx.proximity_upper(), full=True)
    _check_prox(P, z)
    avimp, sqsd, qimp, qimpm = ctx.varimp(True)
    assert np.array_equal(avimp, z["importances"]) and np.array_equal(sqsd, z["sqsd"])
    assert np.array_equal(qimp, z["qimp"])
    assert np.array_equal(ctx.localimp(qimp, qimpm), z["local_importance"])
    votes = ctx.predict_votes(z["Xtest"])
    assert np.array_equal(np.argmax(votes, axis=1).astype(np.int32), z["pred_test"])
    assert np.array_equal(votes.astype(np.float32) / np.float32(f.ntree), z["proba_test"])
    C, _ = ctx.mds3d_full(P)
    rms, scale = _procrustes(C, z["mds3d"])
    assert rms <= 1e-6 * scale, (rms, scale)
    ctx.close()


@pytest.mark.gpu
def test_config1_pybind_mirror_matches_reference(built):
    """The drop-in classifier on config 1: fit grows the forest with the
    library's grower (the reference's forest, see above) and every getter
    returns the reference's arrays."""
    from rfx_b200 import _rfx as rfx

    z, _ = _config1()
    n, p = z["X"].shape
    m = rfx.RandomForestClassifier(nsample=n, ntree=int(z["ntree"]), mdim=p, mtry=int(z["mtry"]), minndsize=1,
                                   compute_proximity=True, compute_importance=True, compute_local_importance=True,
                                   use_gpu=True, show_progress=False)
    m.fit(z["X"], z["y"])
    assert np.float32(m.get_oob_error()) == z["oob_error"]
    assert np.array_equal(m.get_oob_predictions(), z["oob_pred"].astype(np.float32))
    assert np.array_equal(m.feature_importances_(), z["importances"])
    assert np.array_equal(m.get_local_importance(), z["local_importance"])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        _check_prox(m.get_proximity_matrix(), z)
        C = m.compute_mds_3d_cpu()
    rms, scale = _procrustes(C, z["mds3d"])
    assert rms <= 1e-6 * scale, (rms, scale)
    assert np.array_equal(m.predict(z["Xtest"]), z["pred_test"])
    assert np.array_equal(m.predict_proba(z["Xtest"]), z["proba_test"])
    m.cleanup()


# ---------------------------------------------------------------------------
# the benchmarked workload
# ---------------------------------------------------------------------------
N2, T2, SUB = 50_000, 1000, 200


def _bench_subset():
    """The bench's forest (bench.cached_forest) and the analysed tree subset."""
    sys.path.insert(0, ROOT)
    import bench
    from oracle import oracle as orc

    X, y, f, _ = bench.cached_forest(N2, T2)
    Ut = bench.tree_pair_updates(X, y, f)
    heavy = np.argsort(-Ut, kind="stable")[:20]
    rest = np.setdiff1d(np.arange(T2), heavy)
    other = np.random.default_rng(2024).choice(rest, SUB - heavy.size, replace=False)
    trees = np.concatenate([heavy, other])
    sub = f.subset(trees.tolist())
    O = orc.analyse(X, y, sub, do_imp=True, impn=True, do_prox=True, want_leaf=True)
    return X, y, sub, O, int(Ut[trees].sum())


@pytest.mark.gpu
def test_bench_workload_matches_oracle(built):
    import torch

    from oracle import oracle as orc
    from rfx_b200 import abi

    X, y, f, O, U = _bench_subset()
    n, p, T = f.n, f.p, f.ntree
    assert int(O["S"].astype(np.int64).sum()) == U
    ctx = abi.Context(0)
    ctx.load(f, X, y)
    leaf = np.zeros((T, n), np.int32)
    q, nout, _ = ctx.route_oob(leaf=leaf)
    assert np.array_equal(leaf, O["leaf"])
    assert np.array_equal(q.astype(np.float32), O["q_raw"]) and np.array_equal(nout, O["nout"])
    avimp, sqsd, qimp, qimpm = ctx.varimp(True)
    assert np.array_equal(avimp, O["avimp"]) and np.array_equal(sqsd, O["sqsd"])
    assert np.array_equal(qimp, O["qimp"]) and np.array_equal(qimpm, O["qimpm"])
    assert np.array_equal(ctx.localimp(qimp, qimpm), orc.localimp(O["qimp"], O["qimpm"], n, p, T))
    dev = torch.device("cuda", 0)
    L = n * (n + 1) // 2
    S = torch.empty(L, dtype=torch.int32, device=dev)
    ctx.proximity_upper(S)
    ctx.synchronize()
    assert ctx.pair_updates() == U
    S_orc = torch.from_numpy(O["S"]).to(dev)
    assert torch.equal(S, S_orc)
    # the same counts through the hub GEMM + row kernel (the bench's 1,000-tree
    # path; 200 trees alone stay below the hub stage's switch-on)
    os.environ["RFX_PAIRS_HUBS"] = "1"
    try:
        S.fill_(-1)
        ctx.proximity_upper(S)
        ctx.synchronize()
    finally:
        del os.environ["RFX_PAIRS_HUBS"]
    assert torch.equal(S, S_orc)
    # finishprox on 2,000 rows: the members of the forest's largest leaves plus
    # seeded others, against the oracle's finishprox of the same rows
    P = torch.empty(L, dtype=torch.float32, device=dev)
    ctx.finishprox(S, P, full=False)
    ctx.synchronize()
    big = []
    for t in range(T):
        lt = O["leaf"][t]
        vals, cnt = np.unique(lt, return_counts=True)
        term = f.nodestatus[f.offs[t] + vals] == -1  # terminal nodes only (node 0 collects excluded rows)
        k = int(np.argmax(np.where(term, cnt, -1)))
        big.append((int(cnt[k]), t, int(vals[k])))
    big.sort(reverse=True)
    rows = set()
    for _, t, v in big[:5]:
        rows.update(np.flatnonzero(O["leaf"][t] == v)[:200].tolist())
    rng = np.random.default_rng(3)
    rows.update(rng.choice(n, 2000, replace=False).tolist())
    I = np.array(sorted(rows)[:2000], np.int64)
    m = I.size
    ii, jj = np.triu_indices(m)
    a, b = I[ii], I[jj]
    upi = a * n - (a * (a - 1)) // 2 + (b - a)
    S_sub = O["S"][upi]
    P_ref = orc.finishprox(S_sub, O["nout"][I], full=False)
    P_sub = P[torch.from_numpy(upi).to(dev)].cpu().numpy()
    assert np.array_equal(P_sub, P_ref)
    del S, S_orc, P
    ctx.close()
