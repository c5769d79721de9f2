"""The allocation-free Toeplitz apply (hb_toeplitz_apply_noalloc) against hb_toeplitz_apply
and against the FP64 oracle.

The entry point serves callers that may not allocate device memory themselves (for
example a reconstruction plugin inside a host application that owns a fixed device
memory budget): its scratch is a device array built into the library.  The test calls
both entry points through the C ABI, twice in a row with different inputs (the shared
scratch keeps the previous call's contents), then at a second size (the built-in twiddle
tables are rewritten) and at the first size again (rewritten back), and compares each
result within the FP32-path tolerance.  One result per size is also compared with the
oracle's Toeplitz apply directly.  This file is collected last so that a failure here
cannot hide others."""
import ctypes

import numpy as np
import pytest
import torch

from hastycompute_b200 import capi, synth
from hastycompute_b200.toeplitz import ToeplitzPlan
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _rel(a, b):
    return (torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item()


def _setup(shape, cuda, seed):
    plan = ToeplitzPlan(shape, cuda)
    rng = np.random.default_rng(seed)
    coords = rng.uniform(-np.pi, np.pi, (3, 3000)).astype(np.float32)
    packed = plan.build_diagonal(torch.from_numpy(coords))
    mul = synth.gaussian_image(shape, seed=seed + 2)
    return plan, coords, packed, mul


def _both(lib, plan, packed, mul_t, x, base, stream):
    """hb_toeplitz_apply and hb_toeplitz_apply_noalloc, both accumulating x-multiplied
    results into a copy of `base`; returns (workspace result, allocation-free result)."""
    nz, ny, nx = plan.shape
    ref = base.clone()
    got = base.clone()
    nb = lib.hb_normal_workspace_bytes(plan._h, 1, 1)
    ws = torch.empty(nb, dtype=torch.uint8, device=x.device)
    capi.check(lib.hb_toeplitz_apply(plan._h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(ref.data_ptr()),
                                     ny * nx, nx, ctypes.c_void_p(mul_t.data_ptr()), 1,
                                     ctypes.c_void_p(packed.data_ptr()), ctypes.c_void_p(ws.data_ptr()), nb,
                                     stream))
    capi.check(lib.hb_toeplitz_apply_noalloc(nz, ny, nx, ctypes.c_void_p(x.data_ptr()),
                                             ctypes.c_void_p(got.data_ptr()), ny * nx, nx,
                                             ctypes.c_void_p(mul_t.data_ptr()), 1,
                                             ctypes.c_void_p(packed.data_ptr()), stream))
    torch.cuda.synchronize()
    return ref, got


def test_noalloc_matches_workspace_entry_point_and_oracle(cuda):
    lib = capi.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    first, second = (32, 16, 64), (96, 96, 16)
    cases = {s: _setup(s, cuda, seed) for s, seed in ((first, 7), (second, 17))}
    for k, shape in enumerate([first, first, second, first]):
        plan, coords, packed, mul = cases[shape]
        mul_t = torch.from_numpy(mul).to(cuda)
        xn = synth.gaussian_image(shape, seed=10 + k)
        x = torch.from_numpy(xn).to(cuda)
        base = torch.zeros_like(x) + k
        ref, got = _both(lib, plan, packed, mul_t, x, base, stream)
        assert _rel(got, ref) < TOL, (k, shape)
        if k in (0, 2):  # once per size: the oracle's apply_addcmul directly
            T = O.toeplitz_diagonal(coords.astype(np.float64), shape)
            want = k + O.toeplitz_apply(xn, T) * mul
            assert O.rel_l2(got.cpu().numpy().astype(np.complex128), want) < TOL, (k, shape)


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    lib = capi.load()
    n = 128  # 16 * 128^3 bytes > HB_NOALLOC_SCRATCH_BYTES
    assert 16 * n ** 3 > capi.HB_NOALLOC_SCRATCH_BYTES
    code = lib.hb_toeplitz_apply_noalloc(n, n, n, ctypes.c_void_p(1), ctypes.c_void_p(1), n * n, n, None, 0,
                                         ctypes.c_void_p(1), None)
    assert code == capi.HB_ERR_WORKSPACE
    assert b"scratch" in lib.hb_last_error()
