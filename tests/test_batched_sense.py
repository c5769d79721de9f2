"""GPU parity of the batched SENSE operators through the NUFFT (outer/inner batches, coil
subsets and randomisation, k-space manipulators) against the FP64 oracle.

Tolerance: NUFFT at tol 1e-6 in FP32, relative L2 <= 1e-5 (2e-5 where a forward and an
adjoint transform are chained)."""
import numpy as np
import pytest
import torch

from hastycompute_b200 import synth
from hastycompute_b200.batched_sense import BatchedSense, BatchedSenseAdjoint, BatchedSenseNormal
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SHAPE = (16, 16, 16)


def _c64(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a).astype(np.complex64)).to(dev)


def _np(t):
    return t.detach().cpu().numpy().astype(np.complex128)


def _setup(cuda, nouter=2, ninner=2, ncoil=5, seed=0):
    rng = np.random.default_rng(seed)
    coords = [rng.uniform(-np.pi, np.pi, (3, 1500 + 300 * o)).astype(np.float32) for o in range(nouter)]
    sm = synth.coil_maps(ncoil, SHAPE, seed=seed + 1)
    x = rng.standard_normal((nouter, ninner) + SHAPE) + 1j * rng.standard_normal((nouter, ninner) + SHAPE)
    kd = [rng.standard_normal((ninner, ncoil, c.shape[1])) + 1j * rng.standard_normal((ninner, ncoil, c.shape[1]))
          for c in coords]
    w = [rng.uniform(0.2, 1.5, c.shape[1]).astype(np.float32) for c in coords]
    return coords, sm, x, kd, w


@pytest.mark.parametrize("manip", [None, "kdata", "weighted", "weighted_kdata"])
def test_batched_normal_with_manipulators(cuda, manip):
    coords, sm, x, kd, w = _setup(cuda)
    op = BatchedSenseNormal([torch.from_numpy(c) for c in coords], _c64(sm, cuda),
                            kdata_vec=[_c64(k, cuda) for k in kd], weights_vec=[torch.from_numpy(v) for v in w],
                            coils=[0, 2, 4, 1], ninner_batches=2, tol=1e-6)
    out = op.apply(_c64(x, cuda), manipulator=manip)
    for o in range(2):
        for i in range(2):
            ref = O.sense_normal_nufft(coords[o], x[o, i], sm, [0, 2, 4, 1],
                                       kdata=kd[o][i] if manip in ("kdata", "weighted_kdata") else None,
                                       weights=w[o] if manip in ("weighted", "weighted_kdata") else None)
            assert O.rel_l2(_np(out[o, i]), ref) < 2e-5


def test_batched_forward_adjoint_and_per_outer_coils(cuda):
    coords, sm, x, kd, w = _setup(cuda, seed=3)
    coils = [[0, 1, 2], [4, 3]]
    fwd = BatchedSense([torch.from_numpy(c) for c in coords], _c64(sm, cuda), coils=coils, ninner_batches=2, tol=1e-6)
    k = fwd.apply(_c64(x, cuda))
    for o in range(2):
        assert tuple(k[o].shape) == (2, 5, coords[o].shape[1])
        for i in range(2):
            ref = O.sense_forward(coords[o], x[o, i], sm, coils[o])
            assert O.rel_l2(_np(k[o][i, coils[o]]), ref) < 1e-5
            unused = [c for c in range(5) if c not in coils[o]]
            assert float(k[o][i, unused].abs().max()) == 0.0
    adj = BatchedSenseAdjoint([torch.from_numpy(c) for c in coords], _c64(sm, cuda), coils=coils, ninner_batches=2,
                              tol=1e-6)
    kin = [_c64(v, cuda) for v in kd]
    img = adj.apply(kin)
    for o in range(2):
        for i in range(2):
            ref = O.sense_adjoint(coords[o], kd[o][i][coils[o]], sm, coils[o])
            assert O.rel_l2(_np(img[o, i]), ref) < 1e-5
    # reinit to one inner batch
    adj.reinit(ninner_batches=1, coils=coils)
    assert tuple(adj.apply([v[:1] for v in kin]).shape) == (2, 1) + SHAPE


def test_coil_randomization(cuda):
    coords, sm, x, kd, w = _setup(cuda, seed=5)
    op = BatchedSenseNormal([torch.from_numpy(c) for c in coords], _c64(sm, cuda), ninner_batches=2, tol=1e-6)
    op.set_coil_randomization(True, 3)
    np.random.seed(11)
    drawn = op.get_coils()
    assert all(len(c) == 3 and len(set(c)) == 3 and max(c) < 5 for c in drawn)
    np.random.seed(11)
    out = op.apply(_c64(x, cuda))
    for o in range(2):
        ref = O.sense_normal_nufft(coords[o], x[o, 1], sm, drawn[o])
        assert O.rel_l2(_np(out[o, 1]), ref) < 2e-5
    with pytest.raises(RuntimeError, match="manipulator"):
        op.apply(_c64(x, cuda), manipulator="other")
    with pytest.raises(RuntimeError, match="kdata_vec"):
        op.apply(_c64(x, cuda), manipulator="kdata")
