"""The allocation-free pair-count entry point (rfx_pair_counts_noalloc).

It exists for callers that cannot allocate device memory when they call in,
such as a serving process that reserves all GPU memory for its own arena at
start-up and forbids cudaMalloc/cudaFree afterwards.  These tests call it
through the C ABI and compare its output with the ordinary entry point
(rfx_proximity_upper_i32) and with the oracle's dense-branch pair counts on
the same leaves, exactly (integer counts), on two calls in a row: the
library's fixed scratch array keeps the first call's contents, so the second
call must not depend on them.  They also check that a call after the first
takes no device memory, that left-out (-1) leaves and the key-table path for
very many leaves per tree give the oracle's counts, and that an index beyond
max_leaves is refused without a fault.  The file is named so that pytest
collects it last.
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

    from oracle import oracle as orc
    from rfx_b200 import abi

    for (seed, n, T, mtry) in ((31, 3000, 40, 7), (32, 1700, 64, 5)):
        n, T, dense, inbag, max_leaves, S_ref = _case(seed, n, T, mtry)
        S_orc, bad = orc.pairs_from_leaves(dense, inbag, max_leaves)
        assert bad == 0 and np.array_equal(S_orc, S_ref)
        leaf_d = torch.from_numpy(dense).cuda()
        inbag_d = torch.from_numpy(inbag).cuda()
        S_d = torch.full((n * (n + 1) // 2,), -7, dtype=torch.int32, device="cuda")
        abi.pair_counts_noalloc(leaf_d, inbag_d, n, T, max_leaves, S_d)
        assert np.array_equal(S_d.cpu().numpy(), S_ref)
        # second call in a row on the same inputs, output buffer refilled with
        # junk; the device's free memory must not change across it
        S_d.fill_(123)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        abi.pair_counts_noalloc(leaf_d, inbag_d, n, T, max_leaves, S_d)
        free1 = torch.cuda.mem_get_info()[0]
        assert free1 == free0
        assert np.array_equal(S_d.cpu().numpy(), S_ref)


def test_noalloc_left_out_leaves_match_oracle():
    """Some (tree, sample) leaves set to -1 (left out), compared with the
    oracle's counts from the same leaves."""
    import torch

    from oracle import oracle as orc
    from rfx_b200 import abi

    n, T, dense, inbag, max_leaves, _ = _case(33, 2500, 48, 7)
    rng = np.random.default_rng(4)
    dense = dense.copy()
    dense[rng.random(dense.shape) < 0.15] = -1
    S_orc, bad = orc.pairs_from_leaves(dense, inbag, max_leaves)
    assert bad == 0
    S_d = torch.zeros(n * (n + 1) // 2, dtype=torch.int32, device="cuda")
    for _ in range(2):
        abi.pair_counts_noalloc(torch.from_numpy(dense).cuda(), torch.from_numpy(inbag).cuda(), n, T, max_leaves,
                                S_d)
        assert np.array_equal(S_d.cpu().numpy(), S_orc)


def test_noalloc_many_leaves_key_table_in_global_memory():
    """max_leaves large enough that a tree's key counters (2 * max_leaves + 1)
    no longer fit in shared memory: the CSR build keeps them in the tree's
    global segment table and a fix-up pass turns the ends back into starts."""
    import torch

    from oracle import oracle as orc
    from rfx_b200 import abi

    n, T = 30000, 12
    rng = np.random.default_rng(9)
    max_leaves = 30000  # 2 * 30000 + 1 keys per tree: beyond 227 KB of 4-byte counters
    # leaves drawn from a skewed set so that some leaves are large
    leaf = (rng.pareto(1.2, size=(T, n)) * 40).astype(np.int64) % 5000
    leaf = (leaf * 6 + rng.integers(0, 6, size=(T, n))).astype(np.int32)
    assert int(leaf.max()) < max_leaves
    inbag = (rng.random((T, n)) < 0.63).astype(np.uint8)
    S_orc, bad = orc.pairs_from_leaves(leaf, inbag, max_leaves)
    assert bad == 0
    S_d = torch.empty(n * (n + 1) // 2, dtype=torch.int32, device="cuda")
    abi.pair_counts_noalloc(torch.from_numpy(leaf).cuda(), torch.from_numpy(inbag).cuda(), n, T, max_leaves, S_d)
    assert np.array_equal(S_d.cpu().numpy(), S_orc)


def test_noalloc_refuses_index_beyond_max_leaves():
    """A leaf index >= max_leaves is reported as RFX_ERR_INVALID (those samples
    are left out, nothing is written out of bounds), and the next valid call
    still gives the oracle's counts."""
    import torch

    from oracle import oracle as orc
    from rfx_b200 import abi

    n, T, dense, inbag, max_leaves, S_ref = _case(31, 3000, 40, 7)
    bad_leaf = dense.copy()
    bad_leaf[3, 17] = max_leaves  # one index past the declared bound
    S_d = torch.zeros(n * (n + 1) // 2, dtype=torch.int32, device="cuda")
    with pytest.raises(abi.RfxError) as ei:
        abi.pair_counts_noalloc(torch.from_numpy(bad_leaf).cuda(), torch.from_numpy(inbag).cuda(), n, T,
                                max_leaves, S_d)
    assert ei.value.status == 1 and "max_leaves" in str(ei.value)
    S_orc, bad = orc.pairs_from_leaves(bad_leaf, inbag, max_leaves)
    assert bad == 1
    assert np.array_equal(S_d.cpu().numpy(), S_orc)
    abi.pair_counts_noalloc(torch.from_numpy(dense).cuda(), torch.from_numpy(inbag).cuda(), n, T, max_leaves, S_d)
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
