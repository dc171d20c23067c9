"""The C-ABI library loads and exports every symbol include/rfx_b200.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

from conftest import ROOT


def test_header_symbols_exported(built):
    from rfx_b200 import abi

    hdr = open(os.path.join(ROOT, "include", "rfx_b200.h")).read()
    declared = sorted(set(re.findall(r"^\s*(?:rfx_status|const char\*)\s+(rfx_\w+)\s*\(", hdr, re.M)))
    assert declared, "no declarations found"
    lib = ctypes.CDLL(abi.LIB_PATH)
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    assert sorted(abi.EXPORTS) == declared


def test_no_device_is_an_error_not_a_fallback(built):
    """Without a CUDA device the context refuses to open (no CPU fallback)."""
    import torch

    from rfx_b200 import abi

    if torch.cuda.is_available():
        return
    try:
        abi.Context(0)
    except abi.RfxError as e:
        assert e.status in (2, 8)
    else:
        raise AssertionError("context opened without a device")


def test_casewise_context_without_device(built):
    """A case-wise context is a supported configuration: without a device it
    fails for the missing device, not for the option."""
    from rfx_b200 import abi

    try:
        abi.Context(0, use_casewise=True)
    except abi.RfxError as e:
        assert e.status in (2, 8)


def test_tuned_shape_names_cover_every_stage_and_shape(built):
    """Every launch shape the autotuner can record has a name in the binding's
    table (stage ids and shape counts as csrc/tune.cu and the launchers use)."""
    from rfx_b200 import abi

    counts = {0: 10, 1: 8, 2: 9, 3: 9, 4: 8, 5: 2, 6: 2, 7: 2, 8: 2}
    for st, k in counts.items():
        assert len(abi.TUNED_SHAPES[st]) == k, st
