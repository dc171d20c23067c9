"""Device-resident forest hand-off (rfx_forest_load_device): a forest left in
device memory in the padded per-tree layout of the reference's GPU grower
(tree t at slots t * maxnode ...), loaded without a host round trip, gives
the same routing, votes, pair counts and importance as the same forest
loaded from compact host arrays, and the oracle's results."""
import numpy as np
import pytest

from rfx_b200 import synth

pytestmark = pytest.mark.gpu


def _padded(f, maxnode):
    """The compact forest laid out in the padded per-tree layout."""
    T = f.ntree
    pad = lambda a, k=1: np.concatenate([np.pad(a[k * f.offs[t]: k * f.offs[t + 1]], (0, k * (maxnode - f.nnode[t])),
                                                constant_values=-9) for t in range(T)])
    out = dict(nodestatus=pad(f.nodestatus), bestvar=pad(f.bestvar), xbestsplit=pad(f.xbestsplit),
               treemap=pad(f.treemap, 2), nodeclass=pad(f.nodeclass))
    if f.catgoleft is not None:
        out["catgoleft"] = pad(f.catgoleft, f.maxcat)
    return out


@pytest.mark.parametrize("catgoleft", [False, True])
def test_device_load_matches_host_load_and_oracle(built, catgoleft):
    import torch

    from oracle import oracle as orc
    from rfx_b200 import abi

    X, y = synth.mixed_cover(1800, seed=51)
    y = np.unique(y, return_inverse=True)[1].astype(np.int32)
    f = abi.grow_forest(X, y, 30, 7, 1, nclass=int(y.max()) + 1, cat=synth.detect_categorical(X))
    if catgoleft:
        rng = np.random.default_rng(8)
        f.catgoleft = (rng.random(f.total_nodes * f.maxcat) < 0.4).astype(np.int32)
    maxnode = 2 * f.n + 1
    O = orc.analyse(X, y, f, want_leaf=True)
    dev = torch.device("cuda", 0)
    arrays = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in _padded(f, maxnode).items()}
    arrays.update(nin=torch.from_numpy(np.ascontiguousarray(f.nin)).to(dev), X=torch.from_numpy(X).to(dev),
                  y=torch.from_numpy(y).to(dev), cat=torch.from_numpy(f.cat).to(dev))
    ctx = abi.Context(0)
    ctx.load_device(f, arrays, maxnode)
    leaf = np.zeros((f.ntree, f.n), np.int32)
    q, nout, _ = ctx.route_oob(leaf=leaf)
    assert np.array_equal(leaf, O["leaf"])
    assert np.array_equal(q.astype(np.float32), O["q_raw"]) and np.array_equal(nout, O["nout"])
    assert np.array_equal(ctx.proximity_upper(), O["S"])
    if not catgoleft:
        avimp, sqsd, qimp, qimpm = ctx.varimp(True)
        assert np.array_equal(avimp, O["avimp"]) and np.array_equal(qimpm, O["qimpm"])
    ctx.close()


def test_device_load_rejects_host_arrays_and_bad_counts(built):
    import torch

    from rfx_b200 import abi

    X, y = synth.mixed_cover(400, seed=52)
    y = np.unique(y, return_inverse=True)[1].astype(np.int32)
    f = abi.grow_forest(X, y, 4, 7, 1, nclass=int(y.max()) + 1, cat=synth.detect_categorical(X))
    maxnode = 2 * f.n + 1
    host = {k: np.ascontiguousarray(v) for k, v in _padded(f, maxnode).items()}
    host.update(nin=np.ascontiguousarray(f.nin), X=X, y=y, cat=f.cat)
    ctx = abi.Context(0)
    with pytest.raises(abi.RfxError) as ei:
        ctx.load_device(f, host, maxnode)
    assert ei.value.status == 1 and "device memory" in str(ei.value)
    dev = {k: torch.from_numpy(v).cuda() for k, v in host.items()}
    with pytest.raises(abi.RfxError) as ei:
        ctx.load_device(f, dev, int(f.nnode.max()) - 1)  # maxnode smaller than a tree
    assert ei.value.status == 7
    ctx.close()
