"""The allocation-free pair-count entry point (rfx_pair_counts_noalloc).

It exists for callers that cannot allocate device memory when they call in,
such as a serving process that reserves all GPU memory for its own arena at
start-up and forbids cudaMalloc/cudaFree afterwards.  These tests call it
through the C ABI and compare its output with the ordinary entry point
(rfx_proximity_upper_i32) on the same forests, exactly (integer counts), on
two calls in a row: the library's fixed scratch array keeps the first call's
contents, so the second call must not depend on them.  The file is named so
that pytest collects it last.
"""
import numpy as np
import pytest

from rfx_b200 import synth

pytestmark = pytest.mark.gpu


def _dense_leaves(f, leaf_nodes):
    """Node ids from rfx_route_oob -> dense terminal index per tree (-1 = not terminal)."""
    out = np.full(leaf_nodes.shape, -1, np.int32)
    max_leaves = 1
    for t in range(f.ntree):
        ns = f.nodestatus[f.offs[t]:f.offs[t + 1]]
        term = ns == -1
        dense = np.cumsum(term) - 1
        node = leaf_nodes[t]
        out[t] = np.where(term[node], dense[node], -1)
        max_leaves = max(max_leaves, int(term.sum()))
    return out, max_leaves


def _case(seed, n, T, mtry):
    from rfx_b200 import abi

    X, y = synth.mixed_cover(n, seed=seed)
    y = np.unique(y, return_inverse=True)[1].astype(np.int32)
    f = abi.grow_forest(X, y, T, mtry, 1, nclass=int(y.max()) + 1, cat=synth.detect_categorical(X))
    ctx = abi.Context(0)
    ctx.load(f, X, y)
    leaf = np.zeros((T, n), np.int32)
    ctx.route_oob(leaf=leaf)
    S_ref = ctx.proximity_upper()
    ctx.close()
    dense, max_leaves = _dense_leaves(f, leaf)
    inbag = (f.nin > 0).astype(np.uint8)
    return n, T, dense, inbag, max_leaves, S_ref


def test_noalloc_matches_entry_point_twice():
    import torch

    from rfx_b200 import abi

    for (seed, n, T, mtry) in ((31, 3000, 40, 7), (32, 1700, 64, 5)):
        n, T, dense, inbag, max_leaves, S_ref = _case(seed, n, T, mtry)
        leaf_d = torch.from_numpy(dense).cuda()
        inbag_d = torch.from_numpy(inbag).cuda()
        S_d = torch.full((n * (n + 1) // 2,), -7, dtype=torch.int32, device="cuda")
        abi.pair_counts_noalloc(leaf_d, inbag_d, n, T, max_leaves, S_d)
        assert np.array_equal(S_d.cpu().numpy(), S_ref)
        # second call in a row on the same inputs, output buffer refilled with junk
        S_d.fill_(123)
        abi.pair_counts_noalloc(leaf_d, inbag_d, n, T, max_leaves, S_d)
        assert np.array_equal(S_d.cpu().numpy(), S_ref)


def test_noalloc_rejects_oversize():
    import torch

    from rfx_b200 import abi

    n, T = 40000, 30  # n above the 32768 limit
    leaf = torch.zeros((T, n), dtype=torch.int32, device="cuda")
    inbag = torch.zeros((T, n), dtype=torch.uint8, device="cuda")
    S = torch.zeros(1, dtype=torch.int32, device="cuda")
    with pytest.raises(abi.RfxError) as ei:
        abi.pair_counts_noalloc(leaf, inbag, n, T, 10, S)
    assert ei.value.status == 1 and "limits" in str(ei.value)
