"""CPU checks of the native boundary: the C-ABI library loads and exports every symbol
include/hasty_b200.h declares; host-side argument validation needs no GPU."""
import ctypes
import os
import re

import pytest

from hastycompute_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    src = open(os.path.join(ROOT, "include", "hasty_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(hb_[a-z0-9_]+)\s*\(", src)))


def test_header_declarations_match_binding():
    assert _declared_functions() == sorted(capi.SIGNATURES)


def test_library_exports_every_declared_symbol():
    lib = capi.load()
    for name in _declared_functions():
        assert hasattr(lib, name), name


def test_sizes_and_errors_without_gpu():
    lib = capi.load()
    assert lib.hb_version() >= 100
    assert lib.hb_size_supported(128, 128, 128) == 1
    assert lib.hb_size_supported(64, 32, 16) == 1
    assert lib.hb_size_supported(96, 96, 96) == 1
    assert lib.hb_size_supported(160, 160, 128) == 1
    assert lib.hb_size_supported(96, 128, 96) == 0
    assert lib.hb_size_supported(80, 80, 80) == 0
    assert lib.hb_size_supported(256, 128, 128) == 0
    h = ctypes.c_void_p()
    assert lib.hb_plan_create(ctypes.byref(h), 12, 16, 16, 0) == capi.HB_ERR_UNSUPPORTED
    assert b"not supported" in lib.hb_last_error()
    assert lib.hb_plan_create(None, 16, 16, 16, 0) == capi.HB_ERR_INVALID
    # NULL plan is rejected before any CUDA call
    assert lib.hb_toeplitz_apply(None, None, None, 0, 0, None, 0, None, None, 0, None) == capi.HB_ERR_INVALID
    assert lib.hb_normal_workspace_bytes(None, 1, 1) == 0


def test_check_raises_with_message():
    lib = capi.load()
    code = lib.hb_plan_create(None, 16, 16, 16, 0)
    with pytest.raises(capi.HastyError, match="NULL"):
        capi.check(code)


def test_function_lambda_runs_a_torchscript_function():
    """HastyInterface.FunctionLambda (the reference's py_interface.cpp:6-15): a TorchScript
    function compiled from source, called as entry(inout, captures), in place."""
    import torch

    from hastycompute_b200.ffi import hasty_interface as hi

    script = "def apply(a: List[Tensor], b: List[Tensor]):\n    for i in range(len(b)):\n        a[i] += b[i]\n"
    a = [torch.zeros(3), torch.ones(2)]
    hi.FunctionLambda(script, "apply", [torch.arange(3.0), torch.full((2,), 2.0)]).apply(a)
    assert torch.equal(a[0], torch.arange(3.0)) and torch.equal(a[1], torch.full((2,), 3.0))
