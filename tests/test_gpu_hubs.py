"""Hub leaves on the tensor cores (hubs.cu): the leaves with the largest
OOB x in-bag products are counted by an exact u8 x u8 -> s32 tcgen05 GEMM into
byte tiles that the row kernel starts from, the other leaves by the row
kernel.  The split must never change a count: S and the pair-update total are
compared with the oracle's dense-branch counts bit for bit, with the hub part
forced on at small n, with few and with many hub leaves (both operand widths,
128 and 256 hub columns), at n not a multiple of the 128 x 256 tile, and for
every launch shape of the row kernel that reads the tiles."""
import numpy as np
import pytest

from rfx_b200 import synth

pytestmark = pytest.mark.gpu


def _forest(n, T, seed, mtry=7):
    from rfx_b200 import abi

    X, y = synth.mixed_cover(n, seed=seed)
    y = np.unique(y, return_inverse=True)[1].astype(np.int32)
    f = abi.grow_forest(X, y, T, mtry, 1, nclass=int(y.max()) + 1, cat=synth.detect_categorical(X))
    return X, y, f


@pytest.mark.parametrize("n,T,seed,hub_min", [(2600, 24, 41, None), (3001, 60, 42, "1"), (5000, 30, 43, "2000"),
                                              (700, 200, 44, "1")])
def test_hub_counts_match_oracle(built, monkeypatch, n, T, seed, hub_min):
    from oracle import oracle as orc
    from rfx_b200 import abi

    X, y, f = _forest(n, T, seed)
    O = orc.analyse(X, y, f, do_imp=False)
    U = int(O["S"].astype(np.int64).sum())
    monkeypatch.setenv("RFX_PAIRS_HUBS", "1")
    if hub_min is not None:
        monkeypatch.setenv("RFX_PAIRS_HUB_MIN", hub_min)
    for shape in range(8):
        monkeypatch.setenv("RFX_TUNE_PAIRS_HUB", str(shape))
        ctx = abi.Context(0)
        ctx.load(f, X, y)
        ctx.route_oob()
        assert np.array_equal(ctx.proximity_upper(), O["S"]), shape
        assert ctx.pair_updates() == U, shape
        # a second call reuses the tiles' buffers
        assert np.array_equal(ctx.proximity_upper(), O["S"]), shape
        ctx.close()


def test_hub_part_on_and_off_agree(built, monkeypatch):
    """The same forest with the tensor-core part off and on (n = 20,000, above
    the default switch-on size): identical S."""
    import torch

    from rfx_b200 import abi

    X, y, f = _forest(20000, 40, 45)
    L = f.n * (f.n + 1) // 2
    out = []
    for flag in ("0", "1"):
        monkeypatch.setenv("RFX_PAIRS_HUBS", flag)
        ctx = abi.Context(0)
        ctx.load(f, X, y)
        ctx.route_oob()
        S = torch.empty(L, dtype=torch.int32, device="cuda")
        ctx.proximity_upper(S)
        ctx.synchronize()
        out.append((S, ctx.pair_updates()))
        ctx.close()
    assert torch.equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]
