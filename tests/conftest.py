import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def built():
    """Native libraries built in-tree (cheap when up to date)."""
    from rfx_b200 import build
    from oracle import oracle

    build.build()
    oracle.build()
    return True


def has_reference():
    from oracle import reference

    return reference.available()


def single_leaf_tree(f, t: int, cls: int):
    """Replace tree t by a single leaf of class cls."""
    from rfx_b200.forest import Forest

    T = f.ntree
    parts = lambda a, k=1: [a[k * f.offs[u]: k * f.offs[u + 1]] for u in range(T)]
    ns, bv, xs, tm, nc = (parts(f.nodestatus), parts(f.bestvar), parts(f.xbestsplit),
                          parts(f.treemap, 2), parts(f.nodeclass))
    ns[t] = np.array([-1], np.int32)
    bv[t] = np.array([0], np.int32)
    xs[t] = np.array([0.0], np.float32)
    tm[t] = np.array([0, 0], np.int32)
    nc[t] = np.array([cls], np.int32)
    nnode = f.nnode.copy()
    nnode[t] = 1
    offs = np.zeros(T + 1, np.int64)
    offs[1:] = np.cumsum(nnode, dtype=np.int64)
    cat = lambda a: np.ascontiguousarray(np.concatenate(a))
    return Forest(f.n, f.p, f.nclass, f.maxcat, nnode, offs, cat(ns), cat(bv), cat(xs), cat(tm), cat(nc),
                  f.nin.copy(), f.cat.copy(), None)
