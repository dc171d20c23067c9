"""The library's forest producer (rfx_grow_forest) against the reference's own
cpu_bootstrap + cpu_growtree: identical trees, bit for bit."""
import numpy as np
import pytest

from rfx_b200 import synth
from conftest import has_reference


@pytest.mark.skipif(not has_reference(), reason="reference library not built")
@pytest.mark.parametrize("name,gen,mtry,minnd,T", [
    ("gauss", lambda: synth.gaussian_classes(500, 13, 3), 3, 1, 16),
    ("cover", lambda: synth.mixed_cover(1200), 7, 1, 12),
    ("cover_minnd5", lambda: synth.mixed_cover(900, seed=5), 7, 5, 12),
    ("gmm", lambda: synth.large_gmm(800, 32), 5, 5, 10),
    # nodes above 4096 samples take the radix-sort path of the split search
    ("gmm_large_nodes", lambda: synth.large_gmm(12000, 32), 5, 5, 3),
    ("cover_large_nodes", lambda: synth.mixed_cover(9000, seed=9), 7, 1, 2),
])
def test_grow_identical(built, name, gen, mtry, minnd, T):
    from oracle import reference as ref
    from rfx_b200 import abi

    X, y = gen()
    R = ref.grow_forest(X, y, T, mtry, minnd)
    G = abi.grow_forest(X, y, T, mtry, minnd, nclass=int(y.max()) + 1)
    for k in ("nnode", "nodestatus", "bestvar", "xbestsplit", "treemap", "nodeclass", "nin"):
        assert np.array_equal(getattr(R, k), getattr(G, k)), k


def test_bootstrap_matches_oracle(built):
    from oracle import oracle as orc
    from rfx_b200 import abi

    X, y = synth.gaussian_classes(257, 5, 3)
    G = abi.grow_forest(X, y, 5, 2, 1)
    for t in range(5):
        assert np.array_equal(G.nin[t], orc.bootstrap(257, t))


def test_grow_threads_deterministic(built):
    from rfx_b200 import abi

    X, y = synth.mixed_cover(800)
    a = abi.grow_forest(X, y, 9, 7, 1, n_threads=1)
    b = abi.grow_forest(X, y, 9, 7, 1, n_threads=4)
    for k in ("offs", "nodestatus", "bestvar", "xbestsplit", "treemap", "nodeclass", "nin"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
