"""Generate the golden fixtures in tests/golden/ by running the REFERENCE's own
CPU code (oracle/_ref/librfxref.so, built by oracle/Makefile from the
reference sources).  Run from the repository root:

    python tests/golden/make_golden.py

Each fixture holds seeded synthetic inputs, the forest the reference grew, and
the reference's outputs for the post-growth path.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402
from oracle import reference as ref  # noqa: E402
from rfx_b200 import synth  # noqa: E402

CASES = {
    # the small plain-method configuration (n=2000, p=13, 3 classes) at n=300, 60 trees
    "gauss_n300_t60": dict(gen=lambda: synth.gaussian_classes(300, 13, 3), mtry=3, minnd=1, T=60),
    # the mixed-type (cover-shaped, categorical one-hot) configuration at n=400, 40 trees
    "cover_n400_t40": dict(gen=lambda: synth.mixed_cover(400), mtry=7, minnd=1, T=40),
}
PERM_NOOBS = [1, 2, 3, 10, 37, 100, 1000, 7357, 18391]

# The plain-method configuration at its full stated shape: n=2000, p=13,
# 3 balanced classes, ntree=500, mtry=3, nodesize 1.  Its n x n proximity
# matrix (16 MB) is too large to commit, so the fixture holds a SHA-256 of the
# reference's float32 proximity matrix, that matrix's row sums and a few
# complete rows; the forest the reference grew is stored in full together
# with its SHA-256 (the library's grower must reproduce it bit for bit), and
# every other output of the reference in full.
CONFIG1 = dict(name="config1_n2000_t500", n=2000, p=13, c=3, T=500, mtry=3, minnd=1)
FOREST_FIELDS = ("nnode", "nodestatus", "bestvar", "xbestsplit", "treemap", "nodeclass", "nin")
PROX_ROWS = [0, 1, 2, 999, 1000, 1998, 1999]


def forest_digest(f) -> str:
    """SHA-256 over the forest arrays in a fixed order and dtype."""
    import hashlib

    h = hashlib.sha256()
    for k in FOREST_FIELDS:
        a = np.ascontiguousarray(getattr(f, k))
        h.update(k.encode())
        h.update(str(a.dtype).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def array_digest(a) -> str:
    import hashlib

    a = np.ascontiguousarray(a)
    return hashlib.sha256(str(a.dtype).encode() + str(a.shape).encode() + a.tobytes()).hexdigest()


def make_config1():
    c = CONFIG1
    X, y = synth.gaussian_classes(c["n"], c["p"], c["c"])
    cat = synth.detect_categorical(X)
    R = ref.fit_capture(X, y, cat, ntree=c["T"], mtry=c["mtry"], minndsize=c["minnd"])
    f = R["forest"]
    P32 = R["prox"].astype(np.float32)
    mds = ref.mds3d(P32, R["nout"])
    rng = np.random.default_rng(5)
    Xt = (X[:200] + rng.normal(0, 0.4, size=X[:200].shape)).astype(np.float32)
    pred, proba = ref.predict(Xt, f)
    np.savez_compressed(
        os.path.join(HERE, c["name"] + ".npz"),
        X=X, y=y, cat=cat, maxcat=np.int32(f.maxcat), nclass=np.int32(f.nclass), ntree=np.int32(c["T"]),
        mtry=np.int32(c["mtry"]), minndsize=np.int32(c["minnd"]), forest_sha256=np.array(forest_digest(f)),
        nnode=f.nnode, nodestatus=f.nodestatus, bestvar=f.bestvar, xbestsplit=f.xbestsplit, treemap=f.treemap,
        nodeclass=f.nodeclass, nin=f.nin,
        q_raw=R["q_raw"], nout=R["nout"], oob_error=np.float32(R["oob_error"]), oob_pred=R["oob_pred"],
        oob_proba=R["oob_proba"], importances=R["importances"], avimp=R["avimp"], sqsd=R["sqsd"],
        qimp=R["qimp"], local_importance=R["qimpm"], prox_sha256=np.array(array_digest(P32)),
        prox_rowsum=P32.astype(np.float64).sum(axis=1), prox_rows_idx=np.array(PROX_ROWS, np.int32),
        prox_rows=P32[PROX_ROWS], mds3d=mds, Xtest=Xt, pred_test=pred, proba_test=proba)
    print("wrote", c["name"], "nodes", int(f.total_nodes))


def main():
    if not ref.available():
        raise SystemExit("reference library not built: make -f oracle/Makefile REF_DIR=<reference checkout> ref")
    for name, c in CASES.items():
        X, y = c["gen"]()
        cat = synth.detect_categorical(X)
        R = ref.fit_capture(X, y, cat, ntree=c["T"], mtry=c["mtry"], minndsize=c["minnd"])
        f = R["forest"]
        P32 = R["prox"].astype(np.float32)  # get_proximity_matrix's float32 copy
        mds = ref.mds3d(P32, R["nout"])
        rng = np.random.default_rng(5)
        Xt = (X[:50] + rng.normal(0, 0.4, size=X[:50].shape)).astype(np.float32)
        Xt[:, cat > 1] = np.round(Xt[:, cat > 1])
        pred, proba = ref.predict(Xt, f)
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"),
            X=X, y=y, cat=cat, maxcat=np.int32(f.maxcat), nclass=np.int32(f.nclass),
            nnode=f.nnode, nodestatus=f.nodestatus, bestvar=f.bestvar, xbestsplit=f.xbestsplit, treemap=f.treemap,
            nodeclass=f.nodeclass, nin=f.nin,
            q_raw=R["q_raw"], nout=R["nout"], oob_error=np.float32(R["oob_error"]), oob_pred=R["oob_pred"],
            oob_proba=R["oob_proba"], importances=R["importances"], avimp=R["avimp"], sqsd=R["sqsd"],
            qimp=R["qimp"], local_importance=R["qimpm"], prox=P32, mds3d=mds, Xtest=Xt, pred_test=pred,
            proba_test=proba)
        print("wrote", name, "nodes", int(f.nnode.sum()))
    perms = {}
    for noob in PERM_NOOBS:
        _, bad = orc.perm(noob)
        assert bad == 0, noob
        perms[f"perm_{noob}"] = ref.permobmr(noob)
    np.savez_compressed(os.path.join(HERE, "permobmr.npz"), **perms)
    print("wrote permobmr")
    make_config1()


if __name__ == "__main__":
    if sys.argv[1:] == ["config1"]:
        make_config1()
    else:
        main()
