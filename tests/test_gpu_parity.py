"""CUDA path (through the C ABI) against the oracle on the same forests.

Bit-exact for leaf ids, votes, nout, OOB summary, pair counts, importance
counts and the float importance sums (the kernels keep the reference's float
operation order); normalised proximity is compared bit-exact as well (FP64
arithmetic in the same order, then rounded to float32), which is stricter than
the 1e-6 relative tolerance the path requires.
"""
import numpy as np
import pytest

from rfx_b200 import synth

pytestmark = pytest.mark.gpu


def _grow(X, y, T, mtry, minnd=1, cat=None):
    from rfx_b200 import abi

    y = np.unique(y, return_inverse=True)[1].astype(np.int32)
    if cat is None:
        cat = synth.detect_categorical(X)
    f = abi.grow_forest(X, y, T, mtry, minnd, nclass=int(y.max()) + 1, cat=cat)
    return X, y, f


def _with_catgoleft(f, seed=0):
    """An imported forest with non-zero categorical go-left tables."""
    rng = np.random.default_rng(seed)
    f.catgoleft = rng.integers(0, 2, size=f.total_nodes * f.maxcat).astype(np.int32)
    return f


def _wide(n, pg, seed):
    """pg pure-noise Gaussian features followed by the 54 cover-shaped ones,
    which carry the labels (so the informative and categorical features sit
    beyond index 256 when pg > 202)."""
    Xc, y = synth.mixed_cover(n, seed=seed)
    Xg = np.random.default_rng(seed).normal(size=(n, pg)).astype(np.float32)
    return np.ascontiguousarray(np.concatenate([Xg, Xc], axis=1)), y


CASES = {
    "gauss": lambda: _grow(*synth.gaussian_classes(500, 13, 3), 40, 3),
    "cover": lambda: _grow(*synth.mixed_cover(2000), 30, 7),
    "cover_minnd5": lambda: _grow(*synth.mixed_cover(1500, seed=11), 25, 7, 5),
    "catgoleft": lambda: (lambda X, y, f: (X, y, _with_catgoleft(f)))(*_grow(*synth.mixed_cover(1200, seed=3), 20, 7)),
    "tiny": lambda: _grow(*synth.gaussian_classes(7, 3, 2, seed=5), 6, 1),
    "uneven": lambda: (lambda d: _grow(d["X"], d["y"], 12, d["mtry"]))(synth.uneven_forests(1, seed=21, n_range=(900, 900))[0]),
    # more than 256 features: permutation importance runs in feature blocks
    "wide_p304": lambda: _grow(*_wide(450, 250, 41), 24, 17),
    "wide_p600": lambda: _grow(*synth.gaussian_classes(320, 600, 4, seed=43), 16, 24),
}


@pytest.fixture(scope="module", params=list(CASES), ids=list(CASES))
def case(request, built):
    from oracle import oracle as orc
    from rfx_b200 import abi

    X, y, f = CASES[request.param]()
    O = orc.analyse(X, y, f, want_leaf=True, want_jtr=True)
    ctx = abi.Context(0)
    ctx.load(f, X, y)
    yield request.param, X, y, f, O, ctx
    ctx.close()


def test_route_votes_nout_leaf(case):
    name, X, y, f, O, ctx = case
    leaf = np.zeros((f.ntree, f.n), np.int32)
    q, nout, _ = ctx.route_oob(leaf=leaf)
    assert np.array_equal(q.astype(np.float32), O["q_raw"])
    assert np.array_equal(nout, O["nout"])
    assert np.array_equal(leaf, O["leaf"])


def test_oob_summary(case):
    from oracle import oracle as orc

    name, X, y, f, O, ctx = case
    ctx.route_oob()
    err, pred, proba = ctx.oob_summary()
    e2, p2, pr2 = orc.oob_summary(O["q_raw"], O["nout"], y)
    assert err == e2
    assert np.array_equal(pred, p2)
    assert np.array_equal(proba, pr2)


def test_pair_counts_exact(case):
    name, X, y, f, O, ctx = case
    S = ctx.proximity_upper()
    assert np.array_equal(S, O["S"])
    # the pair-update count equals the sum of the strict upper triangle
    assert ctx.pair_updates() == int(O["S"].astype(np.int64).sum())


def test_pair_counts_idempotent(case):
    name, X, y, f, O, ctx = case
    a = ctx.proximity_upper()
    b = ctx.proximity_upper()
    assert np.array_equal(a, b)


def test_finishprox_full_and_upper(case):
    from oracle import oracle as orc

    name, X, y, f, O, ctx = case
    S = ctx.proximity_upper()
    P = ctx.finishprox(S, full=True)
    assert np.array_equal(P, orc.finishprox(O["S"], O["nout"], full=True))
    Pu = ctx.finishprox(S, full=False)
    assert np.array_equal(Pu, orc.finishprox(O["S"], O["nout"], full=False))


def test_varimp_exact(case):
    from oracle import oracle as orc

    name, X, y, f, O, ctx = case
    assert O["perm_bad"] == 0
    avimp, sqsd, qimp, qimpm = ctx.varimp(impn=True)
    assert np.array_equal(avimp, O["avimp"], equal_nan=True)
    assert np.array_equal(sqsd, O["sqsd"], equal_nan=True)
    assert np.array_equal(qimp, O["qimp"])
    assert np.array_equal(qimpm, O["qimpm"])
    li = ctx.localimp(qimp, qimpm)
    assert np.array_equal(li, orc.localimp(O["qimp"], O["qimpm"], f.n, f.p, f.ntree))


def test_varimp_overall_only(case):
    name, X, y, f, O, ctx = case
    avimp, sqsd, qimp, qimpm = ctx.varimp(impn=False)
    assert np.array_equal(avimp, O["avimp"], equal_nan=True)
    assert qimp is None and qimpm is None


def test_predict(case):
    from oracle import oracle as orc

    name, X, y, f, O, ctx = case
    rng = np.random.default_rng(1)
    m = max(3, f.n // 3)
    Xt = (X[:m] + rng.normal(0, 0.5, size=X[:m].shape)).astype(np.float32)
    Xt[:, f.cat > 1] = np.round(Xt[:, f.cat > 1])
    votes = ctx.predict_votes(Xt)
    v2, _, _ = orc.predict(Xt, f)
    assert np.array_equal(votes, v2)


def test_device_outputs_match_host(case):
    import torch

    name, X, y, f, O, ctx = case
    L = f.n * (f.n + 1) // 2
    Sd = torch.empty(L, dtype=torch.int32, device="cuda")
    ctx.proximity_upper(Sd)
    ctx.synchronize()
    assert np.array_equal(Sd.cpu().numpy(), O["S"])
    Pd = torch.empty((f.n, f.n), dtype=torch.float32, device="cuda")
    ctx.finishprox(Sd, Pd, full=True)
    ctx.synchronize()
    from oracle import oracle as orc

    assert np.array_equal(Pd.cpu().numpy(), orc.finishprox(O["S"], O["nout"], full=True))


def test_status2_nodes_route_and_prox(built):
    """Trees holding created-but-unsplit nodes (status 2): testreebag stops on
    them, find_terminal_node walks through them back to the root, and neither
    kind of sample enters the pair counts.  cpu_testreeimp walks through them
    without assigning a vote (the reference keeps a stale value), which the
    library reports instead of guessing."""
    from oracle import oracle as orc
    from rfx_b200 import abi

    X, y, f = _grow(*synth.gaussian_classes(300, 6, 3, seed=8), 8, 2)
    rng = np.random.default_rng(0)
    ns = f.nodestatus.copy()
    for t in range(f.ntree):
        o = f.offs[t]
        leaves = np.flatnonzero(ns[o:f.offs[t + 1]] == -1)
        pick = rng.choice(leaves, size=max(1, leaves.size // 4), replace=False)
        ns[o + pick] = 2
        f.treemap[2 * (o + pick)] = 0
        f.treemap[2 * (o + pick) + 1] = 0
    f.nodestatus = ns
    O = orc.analyse(X, y, f, do_imp=False, want_leaf=True)
    ctx = abi.Context(0)
    ctx.load(f, X, y)
    leaf = np.zeros((f.ntree, f.n), np.int32)
    q, nout, _ = ctx.route_oob(leaf=leaf)
    assert np.array_equal(q.astype(np.float32), O["q_raw"])
    assert np.array_equal(leaf, O["leaf"])
    assert np.array_equal(ctx.proximity_upper(), O["S"])
    with pytest.raises(abi.RfxError) as ei:
        ctx.varimp(impn=True)
    assert ei.value.status == 5
    ctx.close()


def test_forest_validation_rejects_bad_children(built):
    from rfx_b200 import abi

    X, y, f = _grow(*synth.gaussian_classes(200, 5, 2, seed=2), 4, 2)
    k = int(np.flatnonzero(f.nodestatus == 1)[0])
    f.treemap[2 * k] = 10 ** 6
    ctx = abi.Context(0)
    with pytest.raises(abi.RfxError) as ei:
        ctx.load(f, X, y)
    assert ei.value.status == 7
    f.treemap[2 * k] = 1
    f.bestvar[k] = 99
    with pytest.raises(abi.RfxError) as ei:
        ctx.load(f, X, y)
    assert ei.value.status == 7
    ctx.close()


def test_window_crossing_rows(built, monkeypatch):
    """Windowed kernel with n above one column window (24,576 columns): rows
    span two windows."""
    from oracle import oracle as orc
    from rfx_b200 import abi

    monkeypatch.setenv("RFX_PAIRS_KERNEL", "windowed")
    X, y = synth.mixed_cover(26000, seed=17)
    X, y, f = _grow(X, y, 6, 7)
    O = orc.analyse(X, y, f, do_imp=False)
    ctx = abi.Context(0)
    ctx.load(f, X, y)
    S = ctx.proximity_upper()
    assert np.array_equal(S, O["S"])
    ctx.close()


def test_many_trees_two_rounds(built, monkeypatch):
    """More trees than one expansion round of the row kernels (512 / 1024
    trees per round): the tuner's pick, and each balanced row kernel forced."""
    from oracle import oracle as orc
    from rfx_b200 import abi

    X, y, f = _grow(*synth.gaussian_classes(700, 6, 3, seed=4, mean_scale=0.7), 1100, 2)
    O = orc.analyse(X, y, f, do_imp=True)
    for shape in (None, 6, 7):
        if shape is not None:
            monkeypatch.setenv("RFX_TUNE_PAIRS", str(shape))
        ctx = abi.Context(0)
        ctx.load(f, X, y)
        assert np.array_equal(ctx.proximity_upper(), O["S"]), shape
        assert ctx.pair_updates() == int(O["S"].astype(np.int64).sum()), shape
        avimp, sqsd, qimp, qimpm = ctx.varimp(True)
        assert np.array_equal(avimp, O["avimp"]) and np.array_equal(qimpm, O["qimpm"]), shape
        ctx.close()


def test_windowed_pair_kernel(built, monkeypatch):
    """The windowed u32 pair kernel (large n or >= 65536 trees) on small cases."""
    from oracle import oracle as orc
    from rfx_b200 import abi

    monkeypatch.setenv("RFX_PAIRS_KERNEL", "windowed")
    for X, y, f in (_grow(*synth.mixed_cover(1800, seed=9), 20, 7), _grow(*synth.gaussian_classes(400, 5, 3), 30, 2)):
        O = orc.analyse(X, y, f, do_imp=False)
        ctx = abi.Context(0)
        ctx.load(f, X, y)
        assert np.array_equal(ctx.proximity_upper(), O["S"])
        assert ctx.pair_updates() == int(O["S"].astype(np.int64).sum())
        ctx.close()


def test_full_size_properties(built):
    """At the config-2 size (n = 50,000, p = 54) with 64 trees: the pair-update
    count equals an independent count from the leaf histograms, the strict
    upper triangle sums to it, every entry is within [0, T], the diagonal is 0,
    and sampled rows match a recount from the per-tree leaf ids."""
    import torch
    from rfx_b200 import abi

    X, y = synth.mixed_cover(50000)
    X, y, f = _grow(X, y, 64, 7)
    ctx = abi.Context(0)
    ctx.load(f, X, y)
    n, T = f.n, f.ntree
    leaf = np.zeros((T, n), np.int32)
    ctx.route_oob(leaf=leaf)
    Sd = torch.empty(n * (n + 1) // 2, dtype=torch.int32, device="cuda")
    ctx.proximity_upper(Sd)
    ctx.synchronize()
    U = ctx.pair_updates()
    # independent count from the leaf histograms
    inbag = f.nin > 0
    U2 = 0
    term = f.nodestatus == -1
    for t in range(T):
        lt = leaf[t]
        ok = term[f.offs[t] + lt]
        no = np.bincount(lt[ok & ~inbag[t]], minlength=f.nnode[t])
        ni = np.bincount(lt[ok & inbag[t]], minlength=f.nnode[t])
        U2 += int((no.astype(np.int64) * ni).sum())
    assert U == U2
    total = int(Sd.to(torch.int64).sum().item())
    assert total == U
    assert int(Sd.min().item()) >= 0 and int(Sd.max().item()) <= T
    rows = [0, 1, 777, n // 2, n - 2, n - 1]
    Sh = Sd.cpu().numpy()
    for i in rows:
        rec = np.zeros(n, np.int64)
        for t in range(T):
            if not ok_leaf(term, f, t, leaf[t][i]):
                continue
            same = (leaf[t] == leaf[t][i]) & (inbag[t] != inbag[t][i])
            rec += same
        off = i * n - i * (i - 1) // 2
        assert np.array_equal(Sh[off: off + (n - i)], (rec[i:] + 0).astype(np.int32) * (np.arange(i, n) > i))
    ctx.close()


def ok_leaf(term, f, t, node):
    return bool(term[f.offs[t] + node])


@pytest.mark.gpu
@pytest.mark.parametrize("stage,count", [("ROUTE", 10), ("PAIRS", 8), ("VWALK", 9), ("ROUTE_LEAF", 9),
                                         ("VSAMPLE", 2)])
def test_every_launch_shape_matches_oracle(built, monkeypatch, stage, count):
    """Each launch shape the autotuner can pick gives the oracle's results."""
    from oracle import oracle as orc
    from rfx_b200 import abi

    X, y = synth.mixed_cover(2600, seed=23)
    X, y, f = _grow(X, y, 9, 7)
    O = orc.analyse(X, y, f, want_leaf=True)
    for shape in range(count):
        monkeypatch.setenv("RFX_TUNE_" + stage, str(shape))
        ctx = abi.Context(0)
        ctx.load(f, X, y)
        q, nout, _ = ctx.route_oob()
        assert np.array_equal(q.astype(np.float32), O["q_raw"]), shape
        # before any pair counts the walk runs over the OOB lists, after them in leaf order
        avimp, sqsd, qimp, qimpm = ctx.varimp(True)
        assert np.array_equal(avimp, O["avimp"]) and np.array_equal(qimpm, O["qimpm"]), shape
        assert np.array_equal(ctx.proximity_upper(), O["S"]), shape
        # a second pass routes in the leaf order of the first one
        assert np.array_equal(ctx.proximity_upper(), O["S"]), shape
        q2, _, _ = ctx.route_oob()
        assert np.array_equal(q2.astype(np.float32), O["q_raw"]), shape
        avimp, sqsd, qimp, qimpm = ctx.varimp(True)
        assert np.array_equal(avimp, O["avimp"]) and np.array_equal(qimpm, O["qimpm"]), shape
        ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["catgoleft", "cover_minnd5"])
def test_child_prefetch_shapes_match_oracle(built, monkeypatch, name):
    """The child-prefetching walks (leaf-order routing shapes 6-8, importance
    walk shapes 6-8) on a forest with non-zero categorical go-left tables and
    on one grown with minndsize 5: the oracle's votes, leaves, importances and
    pair counts, in natural and in leaf order."""
    from oracle import oracle as orc
    from rfx_b200 import abi

    X, y, f = CASES[name]()
    O = orc.analyse(X, y, f, want_leaf=True)
    for shape in (6, 7, 8):
        monkeypatch.setenv("RFX_TUNE_VWALK", str(shape))
        monkeypatch.setenv("RFX_TUNE_ROUTE_LEAF", str(shape))
        ctx = abi.Context(0)
        ctx.load(f, X, y)
        ctx.route_oob()
        assert np.array_equal(ctx.proximity_upper(), O["S"]), shape
        # routing and the walk now run in the leaf order of the pass above
        leaf = np.zeros((f.ntree, f.n), np.int32)
        q, nout, _ = ctx.route_oob(leaf=leaf)
        assert np.array_equal(q.astype(np.float32), O["q_raw"]), shape
        assert np.array_equal(leaf, O["leaf"]), shape
        assert np.array_equal(ctx.proximity_upper(), O["S"]), shape
        avimp, sqsd, qimp, qimpm = ctx.varimp(True)
        assert np.array_equal(avimp, O["avimp"]) and np.array_equal(sqsd, O["sqsd"]), shape
        assert np.array_equal(qimp, O["qimp"]) and np.array_equal(qimpm, O["qimpm"]), shape
        ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("p", [70, 130, 250])
def test_sample_sum_shapes_multiword_flips(built, monkeypatch, p):
    """Both launch shapes of the per-sample importance sums with two, three
    and four 64-bit flip words per (tree, sample): the oracle's qimp, qimpm,
    avimp and sqsd."""
    from oracle import oracle as orc
    from rfx_b200 import abi

    X, y, f = _grow(*synth.gaussian_classes(600, p, 3, seed=p), 10, max(2, int(np.sqrt(p))))
    O = orc.analyse(X, y, f)
    for shape in (0, 1):
        monkeypatch.setenv("RFX_TUNE_VSAMPLE", str(shape))
        ctx = abi.Context(0)
        ctx.load(f, X, y)
        for _ in range(2):  # over the OOB lists, then in leaf order after the pair counts
            avimp, sqsd, qimp, qimpm = ctx.varimp(True)
            assert np.array_equal(avimp, O["avimp"]) and np.array_equal(sqsd, O["sqsd"]), (p, shape)
            assert np.array_equal(qimp, O["qimp"]) and np.array_equal(qimpm, O["qimpm"]), (p, shape)
            ctx.proximity_upper()
        ctx.close()
