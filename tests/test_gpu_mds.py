"""Full-matrix classical MDS (rfx_mds3d_full) against the reference's own
compute_mds_3d_cpu (LAPACK dsyevd), through the golden fixtures and through
the reference library on a larger forest.  Coordinates are compared after an
orthogonal Procrustes alignment (eigenvectors are defined up to sign, and up to
rotation inside a repeated eigenvalue): RMS <= 1e-6 x the coordinates' RMS."""
import glob
import os

import numpy as np
import pytest

from conftest import ROOT, has_reference
from test_golden import FILES, load

pytestmark = pytest.mark.gpu


def procrustes_rms(C, R):
    U, _, Vt = np.linalg.svd(C.T @ R)
    A = C @ (U @ Vt)
    return float(np.sqrt(np.mean((A - R) ** 2))), float(np.sqrt(np.mean(R ** 2)))


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f)[:-4] for f in FILES])
def test_mds_full_matches_reference_golden(built, path):
    from rfx_b200 import abi

    z, f = load(path)
    ctx = abi.Context(0)
    ctx.load(f, z["X"], z["y"])
    ctx.route_oob()
    S = ctx.proximity_upper()
    P = ctx.finishprox(S, full=True)
    assert np.array_equal(P, z["prox"])
    C, ev = ctx.mds3d_full(P)
    rms, scale = procrustes_rms(C, z["mds3d"])
    assert rms <= 1e-6 * scale, (rms, scale)
    # each column matches up to sign when the eigenvalues are separated
    ctx.close()


@pytest.mark.skipif(not has_reference(), reason="reference library not built")
def test_mds_full_matches_reference_n1500(built):
    from oracle import reference as ref
    from rfx_b200 import abi, synth

    X, y = synth.gaussian_classes(1500, 13, 3, seed=77)
    f = abi.grow_forest(X, y, 80, 3, 1, nclass=3, cat=synth.detect_categorical(X))
    ctx = abi.Context(0)
    ctx.load(f, X, y)
    _, nout, _ = ctx.route_oob()
    P = ctx.finishprox(ctx.proximity_upper(), full=True)
    C, ev = ctx.mds3d_full(P)
    R = ref.mds3d(P, nout)
    rms, scale = procrustes_rms(C, R)
    assert rms <= 1e-6 * scale, (rms, scale)
    ctx.close()
