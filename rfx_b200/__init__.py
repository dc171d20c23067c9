"""rfx_b200 — B200-native (sm_100a) post-growth analysis path of RFX random forests.

The native pieces are ``librfx_b200.so`` (C ABI, include/rfx_b200.h) and the
pybind11 module ``_rfx`` that mirrors the reference's ``rfx`` module surface
(``RandomForestClassifier``, ``confusion_matrix``, ``cuda_is_available``,
``TaskType``), so ``import rfx_b200 as rfx`` reads like code written for ``rfx``.
Both are built in-tree by :mod:`rfx_b200.build`.
"""
from .forest import Forest  # noqa: F401

__all__ = ["Forest", "RandomForestClassifier", "confusion_matrix", "cuda_is_available", "TaskType"]


def __getattr__(name):
    if name in ("RandomForestClassifier", "confusion_matrix", "cuda_is_available", "TaskType"):
        from . import _rfx  # the native module; raises ImportError if it was not built

        return getattr(_rfx, name)
    raise AttributeError(name)
