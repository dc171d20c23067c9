"""Many uneven forests analysed by one captured CUDA graph
(rfx_graph_capture_batch / rfx_graph_launch): every output of every forest
equals the one-forest entry points' output, bit for bit, on two replays."""
import numpy as np
import pytest

from rfx_b200 import synth


def _forests(count=4):
    specs = synth.uneven_forests(count, seed=11, n_range=(600, 3500), p_range=(8, 70), c_range=(2, 9))
    from rfx_b200 import abi

    out = []
    for k, sp in enumerate(specs):
        T = 12 + 7 * k
        f = abi.grow_forest(sp["X"], sp["y"], T, sp["mtry"], 1, nclass=int(sp["y"].max()) + 1)
        out.append((sp["X"], sp["y"], f))
    return out


@pytest.mark.gpu
def test_batch_graph_matches_single_forest_calls(built):
    import torch

    from oracle import oracle as orc
    from rfx_b200 import abi

    dev = torch.device("cuda", 0)
    forests = _forests()
    ctxs, items, ref = [], [], []
    for X, y, f in forests:
        n, p, c = f.n, f.p, f.nclass
        # the one-forest entry points, on their own context
        e = abi.Context(0)
        e.load(f, X, y)
        q, nout, _ = e.route_oob()
        err, pred, _ = e.oob_summary()
        S = e.proximity_upper()
        av, sq, qi, qm = e.varimp(True)
        ref.append(dict(votes=q, nout=nout, oob_error=np.float32(err), oob_pred=pred, S=S, avimp=av, sqsd=sq,
                        qimp=qi, qimpm=qm))
        e.close()
        ctx = abi.Context(0)
        ctx.load(f, X, y)
        ctxs.append(ctx)
        items.append(dict(ctx=ctx, impn=True,
                          votes=torch.zeros(n * c, dtype=torch.int32, device=dev),
                          nout=torch.zeros(n, dtype=torch.int32, device=dev),
                          oob_error=torch.zeros(1, dtype=torch.float32, device=dev),
                          oob_pred=torch.zeros(n, dtype=torch.int32, device=dev),
                          S=torch.zeros(n * (n + 1) // 2, dtype=torch.int32, device=dev),
                          avimp=torch.zeros(p, dtype=torch.float32, device=dev),
                          sqsd=torch.zeros(p, dtype=torch.float32, device=dev),
                          qimp=torch.zeros(n, dtype=torch.float32, device=dev),
                          qimpm=torch.zeros(n * p, dtype=torch.float32, device=dev)))
    # one forest also against the oracle
    X0, y0, f0 = forests[0]
    O = orc.analyse(X0, y0, f0)
    assert np.array_equal(ref[0]["S"], O["S"]) and np.array_equal(ref[0]["avimp"], O["avimp"])

    g = abi.BatchGraph(items)
    assert g.kernel_nodes >= 8 * len(items)
    for rep in range(2):
        for it in items:
            for key in abi.BatchGraph.KEYS:
                it[key].zero_()
        torch.cuda.synchronize()
        g.launch()
        torch.cuda.synchronize()
        for it, r in zip(items, ref):
            assert np.array_equal(it["votes"].cpu().numpy().reshape(r["votes"].shape), r["votes"])
            assert np.array_equal(it["nout"].cpu().numpy(), r["nout"])
            assert it["oob_error"].cpu().numpy()[0] == r["oob_error"]
            assert np.array_equal(it["oob_pred"].cpu().numpy(), r["oob_pred"])
            assert np.array_equal(it["S"].cpu().numpy(), r["S"])
            for key in ("avimp", "sqsd", "qimp", "qimpm"):
                assert np.array_equal(it[key].cpu().numpy().ravel(), np.asarray(r[key]).ravel()), key
    # a reloaded context invalidates the graph
    X, y, f = forests[1]
    ctxs[1].load(f, X, y)
    with pytest.raises(abi.RfxError) as ei:
        g.launch()
    assert ei.value.status == 4
    g.close()
    for c in ctxs:
        c.close()


@pytest.mark.gpu
def test_batch_graph_rejects_host_outputs(built):
    from rfx_b200 import abi

    X, y, f = _forests(1)[0]
    ctx = abi.Context(0)
    ctx.load(f, X, y)
    with pytest.raises(abi.RfxError) as ei:
        abi.BatchGraph([dict(ctx=ctx, S=np.zeros(f.n * (f.n + 1) // 2, np.int32))])
    assert ei.value.status == 1
    ctx.close()
