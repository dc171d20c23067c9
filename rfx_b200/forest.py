"""Compact forest container and its on-disk export format.

The reference keeps every tree padded to ``maxnode = 2n+1`` slots
(src/rf_random_forest.cpp:326-335: ``nodestatus_, bestvar_, xbestsplit_,
treemap_, nodeclass_, catgoleft_`` are all ``ntree * maxnode`` long).  Here a
forest is stored compactly: tree ``t`` owns nodes ``offs[t] .. offs[t+1]``.
Node semantics are the reference's, 0-based:

* ``nodestatus``: -1 terminal, 1 split, 2 created but never split;
* ``treemap[2*node + {0,1}]``: left / right child (node ids local to the tree);
* ``bestvar`` / ``xbestsplit``: split feature and threshold (go left iff
  ``x <= xbestsplit``);
* ``nodeclass``: class of a terminal node;
* ``catgoleft`` (optional, ``maxcat`` ints per node): categorical go-left
  table.  The reference's CPU grower never writes it (src/rf_growtree.cpp:408),
  so ``None`` means all zero.

``nin`` (T x n) holds the bootstrap multiplicity of every sample in every tree.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np

FORMAT_VERSION = 1


@dataclass
class Forest:
    n: int
    p: int
    nclass: int
    maxcat: int
    nnode: np.ndarray          # int32 [T]
    offs: np.ndarray           # int64 [T+1]
    nodestatus: np.ndarray     # int32 [N]
    bestvar: np.ndarray        # int32 [N]
    xbestsplit: np.ndarray     # float32 [N]
    treemap: np.ndarray        # int32 [2N]
    nodeclass: np.ndarray      # int32 [N]
    nin: np.ndarray            # int32 [T, n]
    cat: np.ndarray            # int32 [p]
    catgoleft: Optional[np.ndarray] = None  # int32 [N * maxcat] or None

    @property
    def ntree(self) -> int:
        return int(self.nnode.shape[0])

    @property
    def total_nodes(self) -> int:
        return int(self.offs[-1])

    @classmethod
    def from_padded(cls, n, p, nclass, maxcat, nnode, nodestatus, bestvar, xbestsplit, treemap,
                    nodeclass, nin, cat, catgoleft=None, maxnode=None) -> "Forest":
        """Compact the reference's padded ``T x maxnode`` arrays."""
        T = int(len(nnode))
        mx = int(maxnode if maxnode is not None else 2 * n + 1)
        nnode = np.asarray(nnode, dtype=np.int32)
        offs = np.zeros(T + 1, dtype=np.int64)
        offs[1:] = np.cumsum(nnode, dtype=np.int64)
        ns = np.asarray(nodestatus).reshape(T, mx)
        bv = np.asarray(bestvar).reshape(T, mx)
        xs = np.asarray(xbestsplit).reshape(T, mx)
        tm = np.asarray(treemap).reshape(T, 2 * mx)
        nc = np.asarray(nodeclass).reshape(T, mx)
        cg = None if catgoleft is None else np.asarray(catgoleft).reshape(T, mx * maxcat)
        take = lambda a, k=1: np.concatenate([a[t, : k * nnode[t]] for t in range(T)]) if T else a[:0, 0]
        return cls(
            n=int(n), p=int(p), nclass=int(nclass), maxcat=int(maxcat), nnode=nnode, offs=offs,
            nodestatus=np.ascontiguousarray(take(ns), dtype=np.int32),
            bestvar=np.ascontiguousarray(take(bv), dtype=np.int32),
            xbestsplit=np.ascontiguousarray(take(xs), dtype=np.float32),
            treemap=np.ascontiguousarray(take(tm, 2), dtype=np.int32),
            nodeclass=np.ascontiguousarray(take(nc), dtype=np.int32),
            nin=np.ascontiguousarray(np.asarray(nin).reshape(T, n), dtype=np.int32),
            cat=np.ascontiguousarray(cat, dtype=np.int32),
            catgoleft=None if cg is None else np.ascontiguousarray(take(cg, maxcat), dtype=np.int32),
        )

    def subset(self, trees) -> "Forest":
        """A forest made of the given trees (in the given order)."""
        trees = list(trees)
        nnode = self.nnode[trees]
        offs = np.zeros(len(trees) + 1, dtype=np.int64)
        offs[1:] = np.cumsum(nnode, dtype=np.int64)
        sl = lambda a, k=1: np.concatenate([a[k * self.offs[t]: k * self.offs[t + 1]] for t in trees])
        return Forest(self.n, self.p, self.nclass, self.maxcat, nnode.astype(np.int32), offs,
                      sl(self.nodestatus), sl(self.bestvar), sl(self.xbestsplit), sl(self.treemap, 2),
                      sl(self.nodeclass), np.ascontiguousarray(self.nin[trees]), self.cat.copy(),
                      None if self.catgoleft is None else sl(self.catgoleft, self.maxcat))

    def save(self, path: str) -> None:
        arrays = dict(
            version=np.int32(FORMAT_VERSION), shape=np.array([self.n, self.p, self.nclass, self.maxcat], np.int64),
            nnode=self.nnode, nodestatus=self.nodestatus, bestvar=self.bestvar, xbestsplit=self.xbestsplit,
            treemap=self.treemap, nodeclass=self.nodeclass, nin=self.nin, cat=self.cat)
        if self.catgoleft is not None:
            arrays["catgoleft"] = self.catgoleft
        np.savez_compressed(path, **arrays)

    @classmethod
    def load(cls, path: str) -> "Forest":
        z = np.load(path)
        if int(z["version"]) != FORMAT_VERSION:
            raise ValueError(f"forest export version {int(z['version'])} is not {FORMAT_VERSION}")
        n, p, nclass, maxcat = (int(v) for v in z["shape"])
        nnode = z["nnode"].astype(np.int32)
        offs = np.zeros(nnode.size + 1, dtype=np.int64)
        offs[1:] = np.cumsum(nnode, dtype=np.int64)
        return cls(n, p, nclass, maxcat, nnode, offs, z["nodestatus"], z["bestvar"], z["xbestsplit"],
                   z["treemap"], z["nodeclass"], z["nin"], z["cat"],
                   z["catgoleft"] if "catgoleft" in z.files else None)
