"""GPU parity of the block singular-value thresholding and of the LLR-regularised ADMM
against the FP64 oracle (numpy SVD; FP64 CG).

Tolerances: SVT relative L2 <= 1e-5 (FP64 singular values, FP32 block update); ADMM after
3 outer x 4 CG iterations <= 1e-4 (FP32 CG arithmetic, as the CG tests)."""
import numpy as np
import pytest
import torch

from hastycompute_b200 import capi, synth
from hastycompute_b200.llr import Normal3DBlocksSVT, Random3DBlocksSVT, admm_llr, svt_blocks, waves_of
from hastycompute_b200.toeplitz import ToeplitzPlan
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _c64(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a).astype(np.complex64)).to(dev)


def _np(t):
    return t.detach().cpu().numpy().astype(np.complex128)


def _lowrank(d0, d1, S, rank, seed, noise=0.05):
    rng = np.random.default_rng(seed)
    basis = rng.standard_normal((rank, d1) + S) + 1j * rng.standard_normal((rank, d1) + S)
    coef = rng.standard_normal((d0, rank)) + 1j * rng.standard_normal((d0, rank))
    x = np.einsum("fr,r...->f...", coef, basis)
    return x + noise * (rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape))


@pytest.mark.parametrize("d0,d1,soft,thresh", [(8, 2, True, 3.0), (20, 5, True, 6.0), (8, 2, False, 3), (32, 1, False, 5)])
def test_svt_blocks_against_numpy_svd(cuda, d0, d1, soft, thresh):
    S = (16, 16, 12)
    x = _lowrank(d0, d1, S, 3, seed=d0 + d1)
    corners = [(0, 0, 0), (8, 0, 4), (0, 8, 8), (8, 8, 0), (4, 4, 4)][:4]
    xt = _c64(x, cuda)
    svt_blocks(xt, corners, (8, 8, 4), thresh, soft)
    ref = O.svt_blocks(x, corners, (8, 8, 4), thresh, soft)
    assert O.rel_l2(_np(xt), ref) < 1e-5
    # voxels outside every block are untouched
    mask = np.ones(S, bool)
    for c in corners:
        mask[c[0]:c[0] + 8, c[1]:c[1] + 8, c[2]:c[2] + 4] = False
    assert np.array_equal(_np(xt)[..., mask], x.astype(np.complex64).astype(np.complex128)[..., mask])


def test_block_operators_and_waves(cuda):
    S = (16, 16, 16)
    x = _lowrank(6, 2, S, 2, seed=3)
    op = Normal3DBlocksSVT((6, 2) + S, (4, 4, 4), (8, 8, 8), block_iter=2, thresh=2.0, soft=True, seed=1)
    xt = _c64(x, cuda)
    op.apply(xt)
    ref = x
    for w in op.last_waves:  # strides < shape: overlapping blocks run in consecutive waves
        assert all(not any(all(abs(a - b) < 8 for a, b in zip(c, d)) for d in w[:i]) for i, c in enumerate(w))
        ref = O.svt_blocks(ref, w, (8, 8, 8), 2.0, True)
    assert O.rel_l2(_np(xt), ref) < 1e-5
    rop = Random3DBlocksSVT((6, 2) + S, 12, (4, 8, 4), thresh=1, soft=False, seed=2)
    xt = _c64(x, cuda)
    rop.apply(xt)
    ref = x
    for w in rop.last_waves:
        ref = O.svt_blocks(ref, w, (4, 8, 4), 1, False)
    assert O.rel_l2(_np(xt), ref) < 1e-5
    assert sum(len(w) for w in rop.last_waves) == 12
    assert waves_of([(0, 0, 0), (1, 1, 1), (8, 8, 8)], (4, 4, 4)) == [[(0, 0, 0), (8, 8, 8)], [(1, 1, 1)]]
    with pytest.raises(RuntimeError, match="fit"):
        svt_blocks(_c64(x, cuda), [(10, 0, 0)], (8, 8, 8), 1.0)
    with pytest.raises(capi.HastyError):
        svt_blocks(_c64(np.zeros((33, 1, 8, 8, 8)), cuda), [(0, 0, 0)], (8, 8, 8), 1.0)


def test_admm_llr_against_oracle(cuda):
    shape, d0, d1, ncoil, rho = (16, 16, 16), 3, 2, 3, 0.5
    rng = np.random.default_rng(4)
    sm = synth.coil_maps(ncoil, shape, seed=5)
    plan = ToeplitzPlan(shape, cuda)
    coords = [rng.uniform(-np.pi, np.pi, (3, 1200)).astype(np.float32) for _ in range(d0)]
    packed = torch.stack([plan.build_diagonal(torch.from_numpy(c).to(cuda)) for c in coords])
    Ts = [O.toeplitz_diagonal(c.astype(np.float64), shape) for c in coords]
    xtrue = _lowrank(d0, d1, shape, 2, seed=6, noise=0.01)
    b0 = np.stack([np.stack([O.sense_normal_toeplitz(xtrue[f, e], sm, Ts[f]) for e in range(d1)]) for f in range(d0)])
    svt = Normal3DBlocksSVT((d0, d1) + shape, (8, 8, 8), (8, 8, 8), block_iter=1, thresh=0.05, soft=True, seed=0)
    x = torch.zeros((d0, d1) + shape, dtype=torch.complex64, device=cuda)
    xg, zg = admm_llr(plan, x, _c64(b0, cuda), _c64(sm, cuda), packed, rho, svt, admm_iters=3, cg_iters=4)
    corners = svt.corners()[0]
    xr, zr = O.admm_llr(lambda f, e: (lambda v: O.sense_normal_toeplitz(v, sm, Ts[f])), b0,
                        np.zeros((d0, d1) + shape), rho, lambda v: O.svt_blocks(v, corners, (8, 8, 8), 0.05, True),
                        admm_iters=3, cg_iters=4)
    assert O.rel_l2(_np(xg), xr) < 1e-4
    assert O.rel_l2(_np(zg), zr) < 1e-4
