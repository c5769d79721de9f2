"""GPU tests of the C++/LibTorch host layer and its TorchScript classes against the oracle."""
import numpy as np
import pytest
import torch

from hastycompute_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.fixture(scope="module")
def ffi(cuda):
    from hastycompute_b200.ffi import hasty_toeplitz

    return hasty_toeplitz


def _np(t):
    return t.detach().cpu().numpy().astype(np.complex128)


def test_normal_nufft_toeplitz_from_coords(ffi, cuda):
    shape = (16, 8, 16)
    rng = np.random.default_rng(0)
    coords = torch.from_numpy(rng.uniform(-np.pi, np.pi, (3, 500)).astype(np.float32)).to(cuda)
    op = ffi.NormalNufftToeplitz(coords, [1, *shape])
    T = O.toeplitz_diagonal(coords.cpu().numpy().astype(np.float64), shape)
    assert O.rel_l2(_np(op.get_diagonal()[0]), T) < 1e-6
    x = torch.from_numpy(synth.gaussian_image((1,) + shape, seed=1)).to(cuda)
    M = tuple(2 * n for n in shape)
    s1 = torch.empty((1,) + M, dtype=torch.complex64, device=cuda)
    s2 = torch.empty_like(s1)
    y = op.apply(x, s1, s2)
    ref = O.toeplitz_apply(_np(x[0]), T)
    assert y.shape == (1,) + shape
    assert y.data_ptr() == s2.data_ptr()  # a view into storage2, as in the reference
    assert O.rel_l2(_np(y[0]), ref) < TOL
    add = torch.ones_like(x)
    mul = torch.from_numpy(synth.gaussian_image((1,) + shape, seed=2)).to(cuda)
    op.apply_addcmul(x, add, mul, s1, s2)
    assert O.rel_l2(_np(add[0]), 1 + ref * _np(mul[0])) < TOL
    xi = x.clone()
    op.apply_inplace(xi, s1, s2)
    assert O.rel_l2(_np(xi[0]), ref) < TOL


def test_sense_normal_toeplitz_from_diagonal(ffi, cuda):
    shape = (16, 16, 16)
    rng = np.random.default_rng(1)
    T = O.toeplitz_diagonal(rng.uniform(-np.pi, np.pi, (3, 700)), shape)
    sm = synth.coil_maps(4, shape, seed=3)
    x = synth.gaussian_image((1,) + shape, seed=4)
    op = ffi.SenseNormalToeplitz(None, [1, *shape], torch.from_numpy(T.astype(np.complex64)).reshape(1, 32, 32, 32).to(cuda))
    out = torch.empty((1,) + shape, dtype=torch.complex64, device=cuda)
    coils = [3, 1, 2]
    op.apply(torch.from_numpy(x).to(cuda), out, torch.from_numpy(sm).to(cuda), coils)
    ref = O.sense_normal_toeplitz(x[0], sm, T, coils)
    assert O.rel_l2(_np(out[0]), ref) < TOL


def test_batched_sense_cpu_tensors_and_cg(ffi, cuda):
    shape = (16, 16, 16)
    rng = np.random.default_rng(2)
    Ts = [O.toeplitz_diagonal(rng.uniform(-np.pi, np.pi, (3, 1500)), shape) for _ in range(2)]
    diags = torch.from_numpy(np.stack(Ts).astype(np.complex64))
    sm = synth.coil_maps(3, shape, seed=5)
    nouter = 3
    didx = [1, 0, 1]
    op = ffi.BatchedSenseNormalToeplitz(diags, torch.from_numpy(sm), didx)
    x = torch.from_numpy(np.stack([synth.gaussian_image((1,) + shape, seed=10 + i) for i in range(nouter)]))
    out = torch.empty_like(x)  # CPU tensors, as the reference's batched operators take
    op.apply(x, out, [[0, 1, 2], [2], [0, 1, 2]])
    for i, cl in enumerate([[0, 1, 2], [2], [0, 1, 2]]):
        ref = O.sense_normal_toeplitz(x[i, 0].numpy(), sm, Ts[didx[i]], cl)
        assert O.rel_l2(out[i, 0].numpy(), ref) < TOL
    # CG through the TorchScript class
    lam = 1e-3
    b = torch.empty_like(x)
    op.apply(x, b, None, lam)
    xs = torch.zeros_like(x).to(cuda)
    iters = op.cg(xs, b.to(cuda), 8, 0.0, lam, None)
    assert list(iters) == [8] * nouter
    for i in range(nouter):
        A = O.regularized(lambda v, i=i: O.sense_normal_toeplitz(v, sm, Ts[didx[i]]), lam)
        xo, _ = O.conjugate_gradient(A, b[i, 0].numpy().astype(np.complex128), iters=8)
        assert O.rel_l2(_np(xs[i, 0]), xo) < 1e-4


def test_batched_sense_reduced_precision_through_the_torchscript_class(ffi, cuda):
    """set_precision("bf16x3") on the TorchScript class: the forward x pass runs on the
    tensor cores (ny = nx = 128); the result stays within 1e-4 of the FP64 oracle."""
    shape = (8, 128, 128)
    rng = np.random.default_rng(4)
    T = O.toeplitz_diagonal(rng.uniform(-np.pi, np.pi, (3, 200)), shape)
    sm = synth.coil_maps(2, shape, seed=7)
    op = ffi.BatchedSenseNormalToeplitz(torch.from_numpy(T[None].astype(np.complex64)), torch.from_numpy(sm), [0])
    op.set_precision("bf16x3")
    with pytest.raises(RuntimeError):
        op.set_precision("fp16")
    x = torch.from_numpy(synth.gaussian_image((1, 1) + shape, seed=8))
    out = torch.empty_like(x)
    op.apply(x, out, [[0, 1]])
    ref = O.sense_normal_toeplitz(x[0, 0].numpy(), sm, T, [0, 1])
    assert O.rel_l2(out[0, 0].numpy(), ref) < 1e-4
    # the single-operator classes take the same switch
    sop = ffi.SenseNormalToeplitz(None, [1] + list(shape), torch.from_numpy(T[None].astype(np.complex64)).to(cuda))
    sop.set_precision("bf16x3")
    xs = x[0].to(cuda)
    outs = torch.empty_like(xs)
    sop.apply(xs, outs, torch.from_numpy(sm).to(cuda), [0, 1])
    assert O.rel_l2(outs[0].cpu().numpy(), ref) < 1e-4
    top = ffi.NormalNufftToeplitz(None, [1] + list(shape), torch.from_numpy(T[None].astype(np.complex64)).to(cuda))
    top.set_precision("bf16x3")
    xi = xs.clone()
    s1 = torch.empty((1,) + tuple(2 * n for n in shape), dtype=torch.complex64, device=cuda)
    s2 = torch.empty_like(s1)
    top.apply_inplace(xi, s1, s2)
    assert O.rel_l2(xi[0].cpu().numpy(), O.toeplitz_apply(x[0, 0].numpy(), T)) < 1e-4


def test_legacy_batched_binding_in_place(ffi, cuda):
    shape = (8, 8, 8)
    rng = np.random.default_rng(3)
    Ts = [O.toeplitz_diagonal(rng.uniform(-np.pi, np.pi, (3, 300)), shape) for _ in range(2)]
    sm = synth.coil_maps(2, shape, seed=6)
    x = np.stack([synth.gaussian_image((1,) + shape, seed=20 + i) for i in range(2)])
    xt = torch.from_numpy(x.copy())
    ffi.batched_sense_toeplitz_diagonals(xt, [[0, 1], [0, 1]], torch.from_numpy(sm),
                                         torch.from_numpy(np.stack(Ts).astype(np.complex64)))
    for i in range(2):
        assert O.rel_l2(xt[i, 0].numpy(), O.sense_normal_toeplitz(x[i, 0], sm, Ts[i])) < TOL


def test_errors_are_runtime_errors(ffi, cuda):
    with pytest.raises(RuntimeError, match="not supported"):
        ffi.SenseNormalToeplitz(None, [1, 12, 16, 16], torch.zeros((1, 24, 32, 32), dtype=torch.complex64, device=cuda))
    op = ffi.SenseNormalToeplitz(None, [1, 8, 8, 8], torch.ones((1, 16, 16, 16), dtype=torch.complex64, device=cuda))
    x = torch.zeros((1, 8, 8, 8), dtype=torch.complex64, device=cuda)
    sm = torch.ones((2, 8, 8, 8), dtype=torch.complex64, device=cuda)
    with pytest.raises(RuntimeError, match="coil index"):
        op.apply(x, torch.empty_like(x), sm, [0, 5])


def test_nufft_and_svt_torchscript_classes(cuda):
    """torch.classes.HastyNufft / HastySVT through the reference-named wrappers."""
    from hastycompute_b200.ffi import hasty_nufft, hasty_svt

    shape, K = (8, 16, 16), 1200
    rng = np.random.default_rng(9)
    coords_np = rng.uniform(-np.pi, np.pi, (3, K)).astype(np.float32)
    coords = torch.from_numpy(coords_np).to(cuda)
    c = rng.standard_normal((2, K)) + 1j * rng.standard_normal((2, K))
    op = hasty_nufft.Nufft(coords, [2, *shape], hasty_nufft.NufftOptions(1, True, 1e-6))
    out = torch.empty((2, *shape), dtype=torch.complex64, device=cuda)
    op.apply(torch.from_numpy(c.astype(np.complex64)).to(cuda), out)
    assert O.rel_l2(_np(out), O.nudft_type1(coords_np, c, shape, +1)) < 1e-5
    nn = hasty_nufft.NufftNormal(coords, [1, *shape], hasty_nufft.NufftOptions(2, False, 1e-6),
                                 hasty_nufft.NufftOptions(1, True, 1e-6))
    x = synth.gaussian_image(shape, seed=10)
    y = torch.empty((1, *shape), dtype=torch.complex64, device=cuda)
    st = torch.empty((1, K), dtype=torch.complex64, device=cuda)
    nn.apply(torch.from_numpy(x[None].astype(np.complex64)).to(cuda), y, st)
    assert O.rel_l2(_np(y[0]) / np.prod(shape), O.explicit_normal(x, coords_np)) < 1e-5
    # a function between the transforms (py_nufft.cpp:96-107): here sample weights applied
    # to the k-space data in place, captured by a TorchScript FunctionLambda
    from hastycompute_b200.ffi import hasty_interface

    w = rng.uniform(0.5, 1.5, K)
    wt = torch.from_numpy(w.astype(np.complex64)).to(cuda)
    scale = hasty_interface.FunctionLambda(
        "def apply(a: List[Tensor], b: List[Tensor]):\n    a[0].mul_(b[0])\n", "apply", [wt])
    nn.apply(torch.from_numpy(x[None].astype(np.complex64)).to(cuda), y, st, scale)
    assert O.rel_l2(_np(y[0]) / np.prod(shape), O.explicit_normal(x, coords_np, weights=w)) < 1e-5
    with pytest.raises(RuntimeError, match="nmodes"):
        op.apply(torch.from_numpy(c.astype(np.complex64)).to(cuda), torch.empty((3, *shape), dtype=torch.complex64,
                                                                              device=cuda))
    # SVT on a CPU tensor (moved to the GPU and back, as the reference moves its blocks)
    v = (rng.standard_normal((6, 2, 16, 16, 16)) + 1j * rng.standard_normal((6, 2, 16, 16, 16))).astype(np.complex64)
    vt = torch.from_numpy(v.copy())
    hasty_svt.Normal3DBlocksSVT().apply(vt, [8, 8, 8], [7, 7, 7], 1, 1.5, True)
    ref = O.svt_blocks(v, [(0, 0, 0), (0, 0, 8), (0, 8, 0), (0, 8, 8), (8, 0, 0), (8, 0, 8), (8, 8, 0), (8, 8, 8)],
                       (7, 7, 7), 1.5, True)
    assert O.rel_l2(vt.numpy().astype(np.complex128), ref) < 1e-5
    hasty_svt.Random3DBlocksSVT().apply(vt, 10, [4, 4, 4], 2, False)  # runs; the corners are internal


@pytest.mark.parametrize("centered", [True, False])
def test_preconditioned_cg_through_torchscript_class(ffi, cuda, centered):
    """ConjugateGradient with a CirculantPreconditionerOp through the TorchScript class runs
    the fused device PCG and matches the oracle's FP64 PCG (opalgs.cpp:50-96 with P)."""
    from hastycompute_b200.toeplitz import ToeplitzPlan

    shape, lam, iters = (16, 16, 16), 1e-2, 8
    rng = np.random.default_rng(9)
    coords = rng.uniform(-np.pi, np.pi, (3, 3000)).astype(np.float32)
    sm = synth.coil_maps(4, shape, seed=10)
    ct, smt = torch.from_numpy(coords).to(cuda), torch.from_numpy(sm).to(cuda)
    pc = ffi.circulant_precond_diagonal(smt, ct, lam)  # centred
    Pfft = torch.fft.ifftshift(pc)  # FFT order: the layout hb_precond_build writes
    P_plan = ToeplitzPlan(shape, cuda).build_preconditioner(ct, smt, lam=lam)
    assert O.rel_l2(Pfft.to(torch.complex128), P_plan.to(torch.complex128)) < 1e-6
    T = O.toeplitz_diagonal(coords.astype(np.float64), shape)
    xtrue = synth.gaussian_image(shape, seed=11)
    A = O.regularized(lambda v: O.sense_normal_toeplitz(v, sm, T), lam)
    b = A(xtrue)
    Pn = Pfft.cpu().numpy().astype(np.float64)
    xo, done = O.conjugate_gradient(A, b, iters=iters, P=lambda r: O.precond_apply(Pn, r))
    op = ffi.BatchedSenseNormalToeplitz(torch.from_numpy(T[None].astype(np.complex64)), smt, [0])
    x = torch.zeros((1, 1) + shape, dtype=torch.complex64, device=cuda)
    bt = torch.from_numpy(b.astype(np.complex64)).reshape((1, 1) + shape).to(cuda)
    its = op.cg(x, bt, iters, 0.0, lam, None, pc if centered else Pfft, centered)
    assert list(its) == [done]
    assert O.rel_l2(_np(x[0, 0]), xo) < 1e-4
