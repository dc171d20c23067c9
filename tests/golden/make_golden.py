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


def main():
    if not ref.available():
        raise SystemExit("reference library not built: make -f oracle/Makefile ref")
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


if __name__ == "__main__":
    main()
