"""GPU parity of the NUFFT (types 1 and 2) and the SENSE forward/adjoint against the FP64
direct NUDFT of the oracle.

Tolerance: the gridding error of the requested tolerance plus FP32 rounding; with
tol = 1e-6 (kernel width 7) the relative L2 error must be <= 1e-5, with tol = 1e-3
(width 4) <= 5e-3 (10x and 5x the requested tolerance)."""
import numpy as np
import pytest
import torch

from hastycompute_b200 import capi, synth
from hastycompute_b200.nufft import CUDANufft, NufftOptions, NufftPlan
from hastycompute_b200.toeplitz import ToeplitzPlan
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _c64(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a).astype(np.complex64)).to(dev)


def _np(t):
    return t.detach().cpu().numpy().astype(np.complex128)


def _coords(K, seed, lo=-np.pi, hi=np.pi):
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, (3, K)).astype(np.float32)


def _rand(shape, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("shape", [(16, 16, 16), (8, 16, 32), (32, 8, 8)])
@pytest.mark.parametrize("tol,bound", [(1e-6, 1e-5), (1e-3, 5e-3)])
def test_type1_type2_against_direct_nudft(cuda, shape, tol, bound):
    K = 2500
    coords = _coords(K, 1)
    plan = NufftPlan(torch.from_numpy(coords).to(cuda), shape, tol=tol, maxbatch=2)
    assert plan.width == int(np.ceil(np.log10(1 / tol))) + 1
    c = _rand((3, K), 2)
    f = plan.type1(_c64(c, cuda))
    ref = O.nudft_type1(coords, c, shape, +1)
    assert O.rel_l2(_np(f), ref) < bound
    fm = _rand((3,) + shape, 3)
    cc = plan.type2(_c64(fm, cuda))
    ref2 = O.nudft_type2(coords, fm, -1)
    assert O.rel_l2(_np(cc), ref2) < bound


@pytest.mark.parametrize("shape", [(32, 16), (8, 64), (64,), (16,)])
def test_lower_dimensional_plans_against_direct_nudft(cuda, shape):
    """The reference's 2-D and 1-D plans (nufft.ixx:72-160): coords [d, K], modes [ntransf, *shape]."""
    d, K = len(shape), 1500
    rng = np.random.default_rng(7)
    coords = rng.uniform(-np.pi, np.pi, (d, K)).astype(np.float32)
    ct = torch.from_numpy(coords).to(cuda)
    plan = NufftPlan(ct, shape, tol=1e-6, maxbatch=2)
    c = _rand((3, K), 8)
    assert O.rel_l2(_np(plan.type1(_c64(c, cuda))), O.nudft_type1(coords, c, shape, +1)) < 1e-5
    fm = _rand((3,) + shape, 9)
    assert O.rel_l2(_np(plan.type2(_c64(fm, cuda))), O.nudft_type2(coords, fm, -1)) < 1e-5
    # the reference-named mirror with nmodes [ntransf, *shape] (default tol 1e-5: bound 10x)
    op = CUDANufft(ct, [2, *shape], NufftOptions.type2())
    out = torch.empty((2, K), dtype=torch.complex64, device=cuda)
    op.apply(_c64(fm[:2], cuda), out)
    assert op.ndim() == d and O.rel_l2(_np(out), O.nudft_type2(coords, fm[:2], -1)) < 1e-4
    with pytest.raises(RuntimeError):
        NufftPlan(ct[:1] if d == 2 else torch.cat([ct, ct]), shape)  # rows must match the dimension


def test_signs_batching_and_periodicity(cuda):
    shape, K = (16, 16, 16), 1800
    coords = _coords(K, 4)
    c = _rand((5, K), 5)
    plan = NufftPlan(torch.from_numpy(coords).to(cuda), shape, tol=1e-6, maxbatch=2)
    # the other sign of each type
    f = plan.type1(_c64(c, cuda), isign=-1)
    assert O.rel_l2(_np(f), O.nudft_type1(coords, c, shape, -1)) < 1e-5
    fm = _rand((2,) + shape, 6)
    assert O.rel_l2(_np(plan.type2(_c64(fm, cuda), isign=+1)), O.nudft_type2(coords, fm, +1)) < 1e-5
    # 5 transforms in batches of 2 equal the transforms one by one
    f5 = _np(plan.type1(_c64(c, cuda)))
    for t in range(5):
        assert O.rel_l2(f5[t], _np(plan.type1(_c64(c[t:t + 1], cuda)))[0]) < 1e-6
    # coordinates are 2*pi periodic
    shifted = coords + np.float32(2 * np.pi) * np.sign(coords).astype(np.float32)
    plan2 = NufftPlan(torch.from_numpy(shifted).to(cuda), shape, tol=1e-6)
    assert O.rel_l2(_np(plan2.type1(_c64(c, cuda))), f5) < 1e-5


def test_type2_is_the_adjoint_of_type1(cuda):
    shape, K = (16, 8, 16), 2000
    coords = _coords(K, 7)
    plan = NufftPlan(torch.from_numpy(coords).to(cuda), shape, tol=1e-6)
    f = _rand(shape, 8)
    c = _rand((1, K), 9)
    lhs = np.vdot(_np(plan.type2(_c64(f, cuda), isign=-1)).ravel(), c.ravel())
    rhs = np.vdot(f.ravel(), _np(plan.type1(_c64(c, cuda), isign=+1)).ravel())
    assert abs(lhs - rhs) / abs(rhs) < 1e-5


def test_samples_on_the_grid_and_edges(cuda):
    # samples exactly on fine-grid points, on +-pi and at the origin
    shape = (16, 16, 16)
    g = np.linspace(-np.pi, np.pi, 9, dtype=np.float32)
    zz, yy, xx = np.meshgrid(g, g[::2], np.float32([0.0, np.pi / 16, -np.pi]), indexing="ij")
    coords = np.stack([zz.ravel(), yy.ravel(), xx.ravel()]).astype(np.float32)
    K = coords.shape[1]
    plan = NufftPlan(torch.from_numpy(coords).to(cuda), shape, tol=1e-6)
    c = _rand((1, K), 10)
    assert O.rel_l2(_np(plan.type1(_c64(c, cuda))), O.nudft_type1(coords, c, shape, +1)) < 1e-5


def test_sense_adjoint_and_forward(cuda):
    shape, K, ncoil = (16, 16, 16), 2200, 5
    coords = _coords(K, 11)
    sm = synth.coil_maps(6, shape, seed=12)
    coils = [0, 2, 3, 5, 1]
    plan = NufftPlan(torch.from_numpy(coords).to(cuda), shape, tol=1e-6, maxbatch=2)
    kd = _rand((ncoil, K), 13)
    out = plan.sense_adjoint(_c64(kd, cuda), _c64(sm, cuda), coils)
    assert O.rel_l2(_np(out), O.sense_adjoint(coords, kd, sm, coils)) < 1e-5
    # accumulate adds to the previous content
    plan.sense_adjoint(_c64(kd, cuda), _c64(sm, cuda), coils, out=out, accumulate=True)
    assert O.rel_l2(_np(out), 2 * O.sense_adjoint(coords, kd, sm, coils)) < 1e-5
    x = synth.gaussian_image(shape, seed=14)
    y = plan.sense_forward(_c64(x, cuda), _c64(sm, cuda), coils)
    assert O.rel_l2(_np(y), O.sense_forward(coords, x, sm, coils)) < 1e-5


def test_nufft_normal_equals_eight_times_toeplitz(cuda):
    """type1(type2(x)) / prod(N) (the reference's explicit normal operator) equals 8x the
    Toeplitz operator built from the same samples (the scaling of compare_normal_methods,
    lib/tests/tests1.cpp:351-549)."""
    shape, K = (16, 16, 16), 3000
    coords = _coords(K, 15)
    x = synth.gaussian_image(shape, seed=16)
    nplan = NufftPlan(torch.from_numpy(coords).to(cuda), shape, tol=1e-6)
    explicit = nplan.type1(nplan.type2(_c64(x, cuda)))[0] / float(np.prod(shape))
    tplan = ToeplitzPlan(shape, cuda)
    packed = tplan.build_diagonal(torch.from_numpy(coords).to(cuda))
    toep = torch.zeros(shape, dtype=torch.complex64, device=cuda)
    tplan.apply_add(_c64(x, cuda), toep, packed)
    assert O.rel_l2(_np(explicit), 8 * _np(toep)) < 1e-5


def test_cudanufft_mirror_and_errors(cuda):
    shape, K = (8, 8, 16), 900
    coords = torch.from_numpy(_coords(K, 17)).to(cuda)
    c = _rand((2, K), 18)
    op = CUDANufft(coords, [2] + list(shape), NufftOptions.type1(tol=1e-6))
    out = torch.empty((2,) + shape, dtype=torch.complex64, device=cuda)
    op.apply(_c64(c, cuda), out)
    assert O.rel_l2(_np(out), O.nudft_type1(coords.cpu().numpy(), c, shape, +1)) < 1e-5
    op2 = CUDANufft(coords, [2] + list(shape), NufftOptions.type2(tol=1e-6))
    kd = torch.empty((2, K), dtype=torch.complex64, device=cuda)
    op2.apply(out, kd)
    assert O.rel_l2(_np(kd), O.nudft_type2(coords.cpu().numpy(), _np(out), -1)) < 1e-5
    with pytest.raises(RuntimeError, match="nmodes"):
        op.apply(_c64(c, cuda), torch.empty((3,) + shape, dtype=torch.complex64, device=cuda))
    # 2 * 5 = 10 is not a compiled fine-grid length
    with pytest.raises(capi.HastyError) as e:
        NufftPlan(coords, (5, 8, 8))
    assert e.value.code == capi.HB_ERR_UNSUPPORTED
    with pytest.raises(capi.HastyError) as e:
        NufftPlan(coords, shape, tol=2.0)
    assert e.value.code == capi.HB_ERR_INVALID
    plan = NufftPlan(coords, shape)
    with pytest.raises(capi.HastyError) as e:
        plan.type1(_c64(c, cuda), isign=0)
    assert e.value.code == capi.HB_ERR_INVALID


@pytest.mark.parametrize("shape", [(16, 16, 16), (8, 16, 32), (32, 32, 32)])
def test_diagonal_through_the_nufft_matches_the_exact_build(cuda, shape):
    """hb_diag_build_nufft (the reference's NUFFT construction, tol 1e-6) against the
    FP64-exact hb_diag_build: complex T and the packed diagonal within 1e-5."""
    coords = torch.from_numpy(_coords(4000, 19)).to(cuda)
    plan = ToeplitzPlan(shape, cuda)
    pe, Te = plan.build_diagonal(coords, want_complex=True)
    pn, Tn = plan.build_diagonal(coords, want_complex=True, method="nufft", tol=1e-6)
    assert O.rel_l2(_np(Tn), _np(Te)) < 1e-5
    assert float((pn - pe).norm() / pe.norm()) < 1e-5
    # against the oracle too
    T = O.toeplitz_diagonal(coords.cpu().numpy().astype(np.float64), shape)
    assert O.rel_l2(_np(Tn), T) < 1e-5
    with pytest.raises(RuntimeError, match="method"):
        plan.build_diagonal(coords, method="fast")


@pytest.mark.parametrize("shape", [(96, 96, 8), (160, 160, 8)])
def test_diagonal_through_the_nufft_rejects_unsupported_grids(cuda, shape):
    """4*96 and 4*160 are not fine-grid lengths of the NUFFT: the build says so."""
    coords = torch.from_numpy(_coords(500, 23)).to(cuda)
    plan = ToeplitzPlan(shape, cuda)
    with pytest.raises(capi.HastyError) as e:
        plan.build_diagonal(coords, method="nufft")
    assert e.value.code == capi.HB_ERR_UNSUPPORTED
