"""The allocation-free Toeplitz apply (hb_toeplitz_apply_noalloc) against hb_toeplitz_apply.

The entry point serves callers that may not allocate device memory themselves (for
example a reconstruction plugin inside a host application that owns a fixed device
memory budget): its scratch is a device array built into the library.  The test calls
both entry points through the C ABI, twice in a row with different inputs (the shared
scratch keeps the previous call's contents), and compares them within the FP32-path
tolerance.  This file is collected last so that a failure here cannot hide others."""
import ctypes

import numpy as np
import pytest
import torch

from hastycompute_b200 import capi, synth
from hastycompute_b200.toeplitz import ToeplitzPlan

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _rel(a, b):
    return (torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item()


def test_noalloc_matches_workspace_entry_point_twice(cuda):
    lib = capi.load()
    shape = (32, 16, 64)
    plan = ToeplitzPlan(shape, cuda)
    rng = np.random.default_rng(7)
    coords = torch.from_numpy(rng.uniform(-np.pi, np.pi, (3, 3000)).astype(np.float32))
    packed = plan.build_diagonal(coords)
    mul = torch.from_numpy(synth.gaussian_image(shape, seed=9)).to(cuda)
    stream = ctypes.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    nz, ny, nx = shape
    for call in range(2):
        x = torch.from_numpy(synth.gaussian_image(shape, seed=10 + call)).to(cuda)
        ref = torch.zeros_like(x) + call
        got = ref.clone()
        # existing entry point (caller workspace), accumulate with a multiplier
        nb = lib.hb_normal_workspace_bytes(plan._h, 1, 1)
        ws = torch.empty(nb, dtype=torch.uint8, device=cuda)
        capi.check(lib.hb_toeplitz_apply(plan._h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(ref.data_ptr()),
                                         ny * nx, nx, ctypes.c_void_p(mul.data_ptr()), 1,
                                         ctypes.c_void_p(packed.data_ptr()), ctypes.c_void_p(ws.data_ptr()), nb,
                                         stream))
        capi.check(lib.hb_toeplitz_apply_noalloc(nz, ny, nx, ctypes.c_void_p(x.data_ptr()),
                                                 ctypes.c_void_p(got.data_ptr()), ny * nx, nx,
                                                 ctypes.c_void_p(mul.data_ptr()), 1,
                                                 ctypes.c_void_p(packed.data_ptr()), stream))
        torch.cuda.synchronize()
        assert _rel(got, ref) < TOL, call


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    lib = capi.load()
    n = 128  # 16 * 128^3 bytes > HB_NOALLOC_SCRATCH_BYTES
    assert 16 * n ** 3 > capi.HB_NOALLOC_SCRATCH_BYTES
    code = lib.hb_toeplitz_apply_noalloc(n, n, n, ctypes.c_void_p(1), ctypes.c_void_p(1), n * n, n, None, 0,
                                         ctypes.c_void_p(1), None)
    assert code == capi.HB_ERR_WORKSPACE
    assert b"scratch" in lib.hb_last_error()
