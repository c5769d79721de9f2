"""GPU parity at the benchmarked configuration, against the FP64 oracle.

128^3 complex64 images, 16 coils, the per-frame interleaved golden-angle kooshball of
2000 spokes x 256 samples (frame 0 of 20), lambda = 1e-3, 15-iteration CG, the flow
phantom of the benchmark.  The diagonal is the FP64-exact build (checked against the
oracle's direct NUDFT at smaller sizes in test_gpu_parity.py).

The oracle is the complex128 torch restatement (``oracle.sense_normal_toeplitz_t`` and the
oracle's CG; pinned to the numpy oracle in tests/test_oracle.py), run on the same GPU:
numpy's FFTs of the 256^3 grid would take minutes per solve.

Tolerances (relative L2):
* one FP32 normal-op apply, every compiled 128^2 plane schedule:    <= 1e-5
* one reduced-precision (BF16 hi+lo tensor-core x pass) apply:     <= 1e-4
* 15-iteration CG, FP32 plan: <= 1e-3 and closer to the FP64 CG than the reference's own
  FP32 CG (``opalgs.cpp:50-96`` with complex64 vectors and vdot, replayed by
  ``oracle/torch_ref.py`` on the GPU), the rule of the CPU-runnable configuration;
* 15-iteration CG, reduced-precision plan: <= 1e-3 and within 1e-4 of the FP32 plan's."""
import numpy as np
import pytest
import torch

from hastycompute_b200 import synth
from hastycompute_b200.toeplitz import ToeplitzPlan
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SHAPE = (128, 128, 128)
NCOIL = 16
LAM = 1e-3
ITERS = 15
# plane-pass schedules compiled for 128^2 planes (the autotuner's candidates; 0 is the default)
N_VARIANTS_128 = 10


@pytest.fixture(scope="module")
def cfg2(cuda):
    plan = ToeplitzPlan(SHAPE, cuda)
    coords = synth.kooshball(2000, 256, frame=0, nframes=20)
    packed, Tg = plan.build_diagonal(torch.from_numpy(coords), want_complex=True)
    sm = torch.from_numpy(synth.coil_maps(NCOIL, SHAPE, seed=1)).to(cuda)
    xtrue = torch.from_numpy(synth.flow_phantom(SHAPE, 2, seed=100)).to(cuda)
    T = Tg.to(torch.complex128)
    sm64 = sm.to(torch.complex128)
    A = O.regularized(lambda v: O.sense_normal_toeplitz_t(v, sm64, T), LAM)
    return dict(plan=plan, packed=packed, Tg=Tg, T=T, sm=sm, sm64=sm64, xtrue=xtrue, A=A)


def test_every_128_plane_schedule_matches_oracle(cfg2, monkeypatch):
    """One 16-coil normal-op apply with each compiled plane schedule (the default mod-4
    split, the parity splits, the mod-8 splits) against the FP64 oracle."""
    plan, x = cfg2["plan"], cfg2["xtrue"][0].contiguous()
    ref = O.sense_normal_toeplitz_t(x, cfg2["sm64"], cfg2["T"])
    errs = {}
    for v in [None] + list(range(N_VARIANTS_128)):
        if v is None:
            monkeypatch.delenv("HB_PLANE_VARIANT", raising=False)
        else:
            monkeypatch.setenv("HB_PLANE_VARIANT", str(v))
        out = torch.empty_like(x)
        plan.sense_normal(x, out, cfg2["sm"], cfg2["packed"])
        errs[v] = O.rel_l2(out, ref)
    print("rel L2 vs FP64 oracle per schedule:", errs)
    assert all(e < 1e-5 for e in errs.values()), errs


def test_config2_cg_matches_oracle(cfg2):
    """Two systems of the 4D-flow batch (two velocity encodings of frame 0, one diagonal),
    b = A x_true + lambda x_true, 15 CG iterations from zero."""
    plan, A = cfg2["plan"], cfg2["A"]
    xtrue = cfg2["xtrue"]
    b64 = torch.stack([A(xtrue[e]) for e in range(2)])
    b = b64.to(torch.complex64)
    x = torch.zeros_like(b)
    status, done = plan.cg(x, b, cfg2["sm"], cfg2["packed"], iters=ITERS, lam=LAM, diag_index=[0, 0])
    assert done == [ITERS, ITERS]
    from oracle import torch_ref as R

    Ar = R.ToeplitzSenseNormalCPU(cfg2["Tg"], cfg2["sm"], lam=LAM)
    for e in range(2):
        xo, n = O.conjugate_gradient(A, b[e], iters=ITERS)
        assert n == ITERS
        xr = torch.zeros((1,) + SHAPE, dtype=torch.complex64, device=b.device)
        R.conjugate_gradient(Ar, b[e].reshape((1,) + SHAPE).clone(), xr, iters=ITERS)
        e_gpu = O.rel_l2(x[e], xo)
        e_ref = O.rel_l2(xr[0], xo)
        print(f"system {e}: this path {e_gpu:.3e}, reference FP32 CG {e_ref:.3e} (vs FP64 CG)")
        assert e_gpu < 1e-3 and e_gpu < e_ref


def test_reduced_precision_plan_matches_oracle(cfg2, cuda):
    """The BF16x3 plan (tensor-core forward x pass) at 128^3 x 16 coils: one apply against
    the FP64 oracle, and the 15-iteration CG against the FP64 CG and the FP32 plan."""
    rp = ToeplitzPlan(SHAPE, cuda, precision="bf16x3")
    x = cfg2["xtrue"][0].contiguous()
    out = torch.empty_like(x)
    rp.sense_normal(x, out, cfg2["sm"], cfg2["packed"])
    rp.wait_status()
    ref = O.sense_normal_toeplitz_t(x, cfg2["sm64"], cfg2["T"])
    e_apply = O.rel_l2(out, ref)
    A = cfg2["A"]
    b = A(cfg2["xtrue"][1]).to(torch.complex64).unsqueeze(0).contiguous()
    xr = torch.zeros_like(b)
    rp.cg(xr, b, cfg2["sm"], cfg2["packed"], iters=ITERS, lam=LAM)
    xf = torch.zeros_like(b)
    cfg2["plan"].cg(xf, b, cfg2["sm"], cfg2["packed"], iters=ITERS, lam=LAM)
    xo, _ = O.conjugate_gradient(A, b[0], iters=ITERS)
    e_cg, e_fp = O.rel_l2(xr[0], xo), O.rel_l2(xr[0], xf[0])
    print(f"bf16x3: apply {e_apply:.3e} vs FP64; CG {e_cg:.3e} vs FP64 CG, {e_fp:.3e} vs FP32 plan")
    assert e_apply < 1e-4
    assert e_cg < 1e-3 and e_fp < 1e-4
