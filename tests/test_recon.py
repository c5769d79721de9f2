"""GPU tests of the reconstruction driver (reconstruct_util.py:23-95, 478-508): k-space data
simulated by the oracle's direct NUDFT, diagonals and right-hand sides through the NUFFT,
CG through the Toeplitz normal operator.

Tolerances: against the oracle's FP64 CG on the same normal equations <= 1e-4 after 10
iterations (FP32 CG, NUFFT at tol 1e-6); the image itself is recovered to <= 2e-2 after
40 iterations (consistent data, well-conditioned random sampling)."""
import numpy as np
import pytest
import torch

from hastycompute_b200 import synth
from hastycompute_b200.recon import diagonals_and_rhs, reconstruct_cg_full
from hastycompute_b200.toeplitz import ToeplitzPlan
from oracle import oracle as O

pytestmark = pytest.mark.gpu
SHAPE = (16, 16, 16)


def _c64(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a).astype(np.complex64)).to(dev)


def _np(t):
    return t.detach().cpu().numpy().astype(np.complex128)


def _data(nouter, ncoil, K, seed, weighted):
    rng = np.random.default_rng(seed)
    coords = [rng.uniform(-np.pi, np.pi, (3, K)).astype(np.float32) for _ in range(nouter)]
    sm = synth.coil_maps(ncoil, SHAPE, seed=seed + 1)
    xt = np.stack([synth.gaussian_image(SHAPE, seed=seed + 2 + o) for o in range(nouter)])
    kd = [O.sense_forward(coords[o].astype(np.float64), xt[o], sm) for o in range(nouter)]
    w = [rng.uniform(0.5, 1.5, K).astype(np.float32) for _ in range(nouter)] if weighted else None
    return coords, sm, xt, kd, w


@pytest.mark.parametrize("weighted", [False, True])
def test_reconstruction_from_kspace(cuda, weighted):
    coords, sm, xt, kd, w = _data(2, 4, 6000, 1, weighted)
    plan = ToeplitzPlan(SHAPE, cuda)
    smt = _c64(sm, cuda)
    packed, rhs = diagonals_and_rhs(plan, [torch.from_numpy(c) for c in coords], [_c64(k, cuda) for k in kd], smt,
                                    weights_vec=None if w is None else [torch.from_numpy(v) for v in w])
    # against the oracle's FP64 CG on the same normal equations
    n = float(np.prod(SHAPE))
    for o in range(2):
        c64 = coords[o].astype(np.float64)
        T = O.psf_circulant(c64, SHAPE, weights=None if w is None else w[o].astype(np.float64))
        T = np.fft.fftn(T)
        wk = kd[o] * (1.0 if w is None else w[o][None])
        b = O.sense_adjoint(c64, wk, sm) / (8 * n)
        assert O.rel_l2(_np(rhs[o]), b) < 1e-5
        xr, _ = O.conjugate_gradient(lambda v: O.sense_normal_toeplitz(v, sm, T), b, iters=10)
        x10, _ = reconstruct_cg_full(plan, packed[o:o + 1], rhs[o:o + 1], smt, iters=10)
        assert O.rel_l2(_np(x10[0]), xr) < 1e-4
    x, done = reconstruct_cg_full(plan, packed, rhs, smt, iters=40)
    assert done == [40, 40]
    for o in range(2):
        assert O.rel_l2(_np(x[o]), xt[o]) < 2e-2


def test_initial_image_scaling_and_preconditioner(cuda):
    coords, sm, xt, kd, w = _data(1, 3, 5000, 7, False)
    plan = ToeplitzPlan(SHAPE, cuda)
    smt = _c64(sm, cuda)
    ct = torch.from_numpy(coords[0]).to(cuda)
    packed, rhs = diagonals_and_rhs(plan, [ct], [_c64(kd[0], cuda)], smt)
    # a multiple of the exact solution of the discrete system is rescaled to it (<x, b> / <x, A x>)
    xs, _ = reconstruct_cg_full(plan, packed, rhs, smt, iters=40)
    x, done = reconstruct_cg_full(plan, packed, rhs, smt, iters=3, images=0.5 * xs, tol=1e-3 * float(rhs.norm()))
    assert O.rel_l2(_np(x[0]), _np(xs[0])) < 1e-3 and done[0] <= 1
    # the preconditioned solve reaches the same image
    P = plan.build_preconditioner(ct, smt)
    xp, _ = reconstruct_cg_full(plan, packed, rhs, smt, precond=[P], iters=40)
    assert O.rel_l2(_np(xp[0]), _np(xs[0])) < 1e-2
