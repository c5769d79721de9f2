"""GPU parity of the circulant preconditioner and of preconditioned CG against the FP64 oracle.

Tolerances: the preconditioner's diagonal goes through a type-1 NUFFT at tol 1e-6 and
FP32 FFTs on the 2x grid, relative L2 <= 1e-4 against the oracle; its apply (FP32 FFTs)
<= 1e-5; PCG after 8 iterations <= 1e-4, as for plain CG."""
import numpy as np
import pytest
import torch

from hastycompute_b200 import synth
from hastycompute_b200.toeplitz import System, ToeplitzPlan
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _c64(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a).astype(np.complex64)).to(dev)


def _np(t):
    return t.detach().cpu().numpy().astype(np.complex128)


def _case(shape, ncoil, K, seed, radial=False):
    rng = np.random.default_rng(seed)
    if radial:
        coords = synth.kooshball(max(8, K // 64), 64).astype(np.float32)
    else:
        coords = rng.uniform(-np.pi, np.pi, (3, K)).astype(np.float32)
    sm = synth.coil_maps(ncoil, shape, seed=seed + 1)
    return coords, sm


@pytest.mark.parametrize("shape", [(16, 16, 16), (8, 16, 32)])
def test_build_and_apply_against_oracle(cuda, shape):
    coords, sm = _case(shape, 4, 3000, 1)
    plan = ToeplitzPlan(shape, cuda)
    lam = 1e-2
    P = plan.build_preconditioner(torch.from_numpy(coords).to(cuda), _c64(sm, cuda), coils=[0, 1, 3], lam=lam)
    ref = O.circulant_precond(coords.astype(np.float64), sm, lam, coils=[0, 1, 3])
    assert O.rel_l2(P.cpu().numpy().astype(np.float64), ref) < 1e-4
    x = synth.gaussian_image(shape, seed=2)
    y = plan.apply_preconditioner(P, _c64(x, cuda))
    Pn = P.cpu().numpy().astype(np.float64)
    assert O.rel_l2(_np(y), O.precond_apply(Pn, x)) < 1e-5
    # in place
    xt = _c64(x, cuda)
    plan.apply_preconditioner(P, xt, out=xt)
    assert O.rel_l2(_np(xt), O.precond_apply(Pn, x)) < 1e-5


def _pcg_case(cuda, shape, ncoil, K, seed, lam, radial=False):
    coords, sm = _case(shape, ncoil, K, seed, radial)
    plan = ToeplitzPlan(shape, cuda)
    ct = torch.from_numpy(coords).to(cuda)
    packed, T = plan.build_diagonal(ct, want_complex=True)
    P = plan.build_preconditioner(ct, _c64(sm, cuda), lam=lam)
    xtrue = synth.gaussian_image(shape, seed=seed + 5)
    Tn = _np(T)
    A = lambda v: O.sense_normal_toeplitz(v, sm, Tn) + lam * v  # noqa: E731
    b = A(xtrue)
    return plan, sm, packed, P, A, b


def test_pcg_matches_oracle_pcg(cuda):
    shape, lam, iters = (16, 16, 16), 1e-2, 8
    plan, sm, packed, P, A, b = _pcg_case(cuda, shape, 4, 3000, 3, lam)
    Pn = P.cpu().numpy().astype(np.float64)
    xr, done = O.conjugate_gradient(A, b, iters=iters, P=lambda r: O.precond_apply(Pn, r))
    x = torch.zeros(shape, dtype=torch.complex64, device=cuda)
    st, it = plan.cg_systems([System(x, _c64(sm, cuda), packed, b=_c64(b, cuda), lam=lam, precond=P)], iters=iters)
    assert it == [done]
    assert O.rel_l2(_np(x), xr) < 1e-4


def test_pcg_converges_faster_on_a_radial_trajectory(cuda):
    shape, lam, iters = (32, 32, 32), 1e-3, 6
    plan, sm, packed, P, A, b = _pcg_case(cuda, shape, 4, 40000, 4, lam, radial=True)
    res = {}
    for name, pc in (("cg", None), ("pcg", P)):
        x = torch.zeros(shape, dtype=torch.complex64, device=cuda)
        plan.cg_systems([System(x, _c64(sm, cuda), packed, b=_c64(b, cuda), lam=lam, precond=pc)], iters=iters)
        res[name] = np.linalg.norm(b - A(_np(x))) / np.linalg.norm(b)
    assert res["pcg"] < 0.7 * res["cg"], res  # measured: 0.20 vs 0.40 after 6 iterations


def test_mixed_batch_graph_and_eager(cuda):
    """Systems with and without a preconditioner share one launch sequence; the plain one
    matches plain CG, the preconditioned one is the same with and without graph replay."""
    shape, lam, iters = (16, 16, 16), 1e-2, 5
    plan, sm, packed, P, A, b = _pcg_case(cuda, shape, 3, 2500, 6, lam)
    smt, bt = _c64(sm, cuda), _c64(b, cuda)
    outs = []
    for graph in (True, False):
        xs = [torch.zeros(shape, dtype=torch.complex64, device=cuda) for _ in range(2)]
        plan.cg_systems([System(xs[0], smt, packed, b=bt, lam=lam, precond=P),
                         System(xs[1], smt, packed, b=bt, lam=lam)], iters=iters, graph=graph)
        outs.append(xs)
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])
    xplain = torch.zeros(shape, dtype=torch.complex64, device=cuda)
    plan.cg_systems([System(xplain, smt, packed, b=bt, lam=lam)], iters=iters)
    assert O.rel_l2(_np(outs[0][1]), _np(xplain)) < 1e-5
    assert O.rel_l2(_np(outs[0][0]), _np(xplain)) > 1e-3  # the preconditioner changed the iterates
