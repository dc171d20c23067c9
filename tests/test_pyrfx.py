"""The pybind11 mirror of the reference's rfx classification API: checks that
need no GPU (module surface, argument validation, confusion_matrix, and that
fitting without a device fails loudly instead of falling back to the CPU)."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def rfx(built):
    from rfx_b200 import _rfx

    return _rfx


def test_surface(rfx):
    for name in ("RandomForestClassifier", "confusion_matrix", "cuda_is_available", "TaskType"):
        assert hasattr(rfx, name)
    C = rfx.RandomForestClassifier
    for meth in ("fit", "predict", "predict_proba", "get_oob_error", "feature_importances_", "get_task_type",
                 "get_n_samples", "get_n_features", "get_n_classes", "get_local_importance", "get_proximity_matrix",
                 "compute_proximity_matrix", "get_oob_predictions", "get_lowrank_factors", "compute_mds_3d_cpu",
                 "compute_mds_from_factors", "compute_mds_3d_from_factors", "cleanup"):
        assert hasattr(C, meth), meth


def test_constructor_defaults_and_validation(rfx):
    m = rfx.RandomForestClassifier()
    assert m.get_task_type() == rfx.TaskType.CLASSIFICATION
    assert m.get_n_samples() == 1000 and m.get_n_features() == 10 and m.get_n_classes() == 2
    # the reference's 31 keyword arguments are all accepted
    rfx.RandomForestClassifier(nsample=10, ntree=5, mdim=3, nclass=2, maxcat=10, mtry=1, maxnode=0, minndsize=1,
                               ncsplit=25, ncmax=25, iseed=7, compute_proximity=True, compute_importance=True,
                               compute_local_importance=True, use_gpu=True, use_qlora=True, quant_mode="INT8",
                               use_sparse=False, sparsity_threshold=1e-6, batch_size=0, nodesize=5, cutoff=0.01,
                               show_progress=False, progress_desc="x", gpu_loss_function="gini", rank=16,
                               n_threads_cpu=2, use_rfgap=False, importance_method="local_imp", clique_M=-1,
                               use_casewise=False)
    with pytest.raises(RuntimeError, match="Unknown quantization level"):
        rfx.RandomForestClassifier(quant_mode="int4")
    with pytest.raises(RuntimeError, match="only be used for regression"):
        rfx.RandomForestClassifier(gpu_loss_function="mse")
    with pytest.raises(RuntimeError, match="Unknown loss function"):
        rfx.RandomForestClassifier(gpu_loss_function="entropy")


def test_unfitted_calls_raise(rfx):
    m = rfx.RandomForestClassifier()
    for call in (lambda: m.predict(np.zeros((2, 10), np.float32)), m.get_oob_error, m.get_oob_predictions,
                 m.get_lowrank_factors, m.compute_mds_3d_cpu, lambda: m.compute_mds_from_factors(3)):
        with pytest.raises(RuntimeError, match="must be fitted"):
            call()
    m.cleanup()  # idempotent
    m.cleanup()


def test_confusion_matrix(rfx):
    rng = np.random.default_rng(0)
    t = rng.integers(0, 4, 500).astype(np.int32)
    p = rng.integers(0, 5, 500).astype(np.int32)
    cm = rfx.confusion_matrix(t, p)
    assert cm.dtype == np.int32 and cm.shape == (5, 5)
    ref = np.zeros((5, 5), np.int32)
    np.add.at(ref, (t, p), 1)
    assert np.array_equal(cm, ref)
    # negative labels are skipped, the size follows the largest label
    cm2 = rfx.confusion_matrix(np.array([0, -1, 2], np.int32), np.array([1, 1, -3], np.int32))
    assert cm2.shape == (3, 3) and cm2.sum() == 1 and cm2[0, 1] == 1


def test_unsupported_options_raise(rfx):
    X = np.zeros((8, 2), np.float32)
    y = np.array([0, 1] * 4, np.int32)
    with pytest.raises(RuntimeError, match="use_rfgap=True with use_qlora=True"):
        rfx.RandomForestClassifier(ntree=2, compute_proximity=True, use_rfgap=True, use_qlora=True).fit(X, y)
    with pytest.raises(RuntimeError, match="CLIQUE"):
        rfx.RandomForestClassifier(ntree=2, compute_local_importance=True, importance_method="clique").fit(X, y)
    with pytest.raises(RuntimeError, match="2-dimensional"):
        rfx.RandomForestClassifier(ntree=2).fit(np.zeros(8, np.float32), y)


def test_no_device_fails_loudly(rfx):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    assert rfx.cuda_is_available() is False
    rng = np.random.default_rng(1)
    X = rng.normal(size=(40, 3)).astype(np.float32)
    y = (X[:, 0] > 0).astype(np.int32)
    m = rfx.RandomForestClassifier(nsample=40, ntree=3, mdim=3, show_progress=False)
    with pytest.raises(RuntimeError, match="CUDA context"):
        m.fit(X, y)


def test_package_reads_like_rfx(built):
    """`import rfx_b200 as rfx` exposes the reference module's names."""
    import rfx_b200 as rfx
    from rfx_b200 import _rfx

    for name in ("RandomForestClassifier", "confusion_matrix", "cuda_is_available", "TaskType"):
        assert getattr(rfx, name) is getattr(_rfx, name)
