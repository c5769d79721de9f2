"""CPU tests of the FP64 oracle: pinned to the reference's own code and known answers."""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden_ahwa.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("case", ["cnm", "rnd"])
def test_toeplitz_matches_reference_dense_builder(golden, case):
    """Oracle Toeplitz op x prod(2N) == the reference's dense A^H W A
    (toep_builder.py compute_AHWA, executed from the reference source by make_golden.py)."""
    x = golden[f"x_{case}"]
    y = golden[f"y_{case}"]
    nf = int(golden[f"nf_{case}"])
    c = golden["coords"][:, :nf].astype(np.float64)
    T = O.toeplitz_diagonal(c, x.shape)
    got = O.toeplitz_apply(x, T) * np.prod(O.grid2(x.shape))
    assert O.rel_l2(got, y) < 1e-12


@pytest.mark.parametrize("case", ["cnm", "rnd"])
def test_explicit_normal_matches_reference_dense_builder(golden, case):
    x = golden[f"x_{case}"]
    y = golden[f"y_{case}"]
    nf = int(golden[f"nf_{case}"])
    c = golden["coords"][:, :nf].astype(np.float64)
    got = O.explicit_normal(x, c) * np.prod(x.shape)
    assert O.rel_l2(got, y) < 1e-12


def test_explicit_over_toeplitz_is_eight(golden):
    """compare_normal_methods (tests1.cpp:351-549): explicit normal / Toeplitz = 2^3."""
    x = golden["x_cnm"]
    c = golden["coords"][:, :30].astype(np.float64)
    T = O.toeplitz_diagonal(c, x.shape)
    ratio = O.explicit_normal(x, c) / O.toeplitz_apply(x, T)
    assert np.allclose(ratio, 8.0, rtol=1e-10, atol=0)


def test_real_part_of_diagonal_suffices():
    rng = np.random.default_rng(3)
    N = (6, 4, 8)
    c = rng.uniform(-np.pi, np.pi, (3, 400))
    T = O.toeplitz_diagonal(c, N)
    assert np.abs(T.imag).max() > 1e-3 * np.abs(T).max()  # Im(T) is not negligible ...
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    a = O.toeplitz_apply(x, T)
    b = O.toeplitz_apply(x, T.real.astype(np.complex128))
    assert O.rel_l2(b, a) < 1e-13  # ... but it never reaches the cropped output


def test_diagonal_build_matches_impulse_construction():
    """nufft.cpp:932-971 literally: impulse at M/2, normal op on the 2x grid, ifftshift, fftn."""
    rng = np.random.default_rng(4)
    N = (4, 6, 4)
    M = O.grid2(N)
    c = rng.uniform(-np.pi, np.pi, (3, 50))
    delta = np.zeros(M, np.complex128)
    delta[M[0] // 2, M[1] // 2, M[2] // 2] = 1.0
    normal = O.explicit_normal(delta, c) * np.prod(M) / np.prod(M)  # explicit on the M grid: /prod(M)
    T_imp = np.fft.fftn(np.fft.ifftshift(normal))
    T = O.toeplitz_diagonal(c, N)
    assert O.rel_l2(T, T_imp) < 1e-12


def _dense(op, shape):
    n = int(np.prod(shape))
    A = np.zeros((n, n), np.complex128)
    for j in range(n):
        e = np.zeros(n, np.complex128)
        e[j] = 1
        A[:, j] = op(e.reshape(shape)).ravel()
    return A


def test_sense_normal_dense_hermitian_psd():
    rng = np.random.default_rng(5)
    N = (4, 4, 4)
    c = rng.uniform(-np.pi, np.pi, (3, 300))
    T = O.toeplitz_diagonal(c, N)
    sm = rng.standard_normal((3,) + N) + 1j * rng.standard_normal((3,) + N)
    A = _dense(lambda v: O.sense_normal_toeplitz(v, sm, T), N)
    assert np.allclose(A, A.conj().T, atol=1e-10 * np.abs(A).max())
    assert np.linalg.eigvalsh(A).min() > -1e-9 * np.abs(A).max()


def test_cg_matches_direct_solve():
    rng = np.random.default_rng(6)
    N = (4, 4, 4)
    c = rng.uniform(-np.pi, np.pi, (3, 500))
    T = O.toeplitz_diagonal(c, N)
    sm = rng.standard_normal((2,) + N) + 1j * rng.standard_normal((2,) + N)
    lam = 1e-1
    op = O.regularized(lambda v: O.sense_normal_toeplitz(v, sm, T), lam)
    A = _dense(op, N)
    b = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    x_direct = np.linalg.solve(A, b.ravel()).reshape(N)
    x, n = O.conjugate_gradient(op, b, iters=200, tol=1e-12)
    assert O.rel_l2(x, x_direct) < 1e-8


def test_cg_not_positive_definite_raises():
    b = np.ones((2, 2, 2), np.complex128)
    with pytest.raises(O.NotPositiveDefinite):
        O.conjugate_gradient(lambda v: -v, b, iters=3)


def test_cg_tol_and_iter_zero():
    b = np.ones((2, 2, 2), np.complex128)
    x, n = O.conjugate_gradient(lambda v: 2 * v, b, iters=0)
    assert n == 0 and np.all(x == 0)
    x, n = O.conjugate_gradient(lambda v: 2 * v, b, iters=10, tol=1e-9)
    assert n == 1 and np.allclose(x, 0.5)


def test_nudft_pair_pinned_to_the_explicit_normal(golden):
    """The direct type-1 / type-2 NUDFTs compose to the explicit normal operator that the
    reference's dense builder pins (type 2 with isign -1, type 1 with isign +1, over
    prod(N)), and type 2 (-1) is the adjoint of type 1 (+1)."""
    x = golden["x_cnm"]
    c = golden["coords"][:, :30].astype(np.float64)
    y = O.nudft_type1(c, O.nudft_type2(c, x, -1), x.shape, +1)[0] / np.prod(x.shape)
    assert O.rel_l2(y, O.explicit_normal(x, c)) < 1e-12
    rng = np.random.default_rng(5)
    f = rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape)
    k = rng.standard_normal((1, 30)) + 1j * rng.standard_normal((1, 30))
    lhs = np.vdot(O.nudft_type2(c, f, -1).ravel(), k.ravel())
    rhs = np.vdot(f.ravel(), O.nudft_type1(c, k, x.shape, +1).ravel())
    assert abs(lhs - rhs) < 1e-10 * abs(rhs)


def test_sense_adjoint_forward_oracle_pair():
    rng = np.random.default_rng(6)
    shape, K = (4, 3, 5), 40
    c = rng.uniform(-np.pi, np.pi, (3, K))
    sm = rng.standard_normal((3,) + shape) + 1j * rng.standard_normal((3,) + shape)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    kd = rng.standard_normal((2, K)) + 1j * rng.standard_normal((2, K))
    coils = [2, 0]
    lhs = np.vdot(O.sense_forward(c, x, sm, coils).ravel(), kd.ravel())
    rhs = np.vdot(x.ravel(), O.sense_adjoint(c, kd, sm, coils).ravel())
    assert abs(lhs - rhs) < 1e-10 * abs(rhs)


def test_circulant_precond_is_the_fourier_diagonal():
    """The preconditioner's d[k] equals the diagonal of F B F^H (F the unitary DFT of the
    N grid, B = sum_c S_c^H Top S_c + lam I), computed here by brute force column by
    column; and P is Hermitian positive definite."""
    rng = np.random.default_rng(7)
    shape, K, lam = (4, 3, 5), 60, 0.3
    c = rng.uniform(-np.pi, np.pi, (3, K))
    sm = rng.standard_normal((2,) + shape) + 1j * rng.standard_normal((2,) + shape)
    T = O.toeplitz_diagonal(c, shape)
    n = int(np.prod(shape))
    d_brute = np.empty(n)
    for k in range(n):
        e = np.zeros(n, np.complex128)
        e[k] = 1.0
        fk = np.fft.ifftn(e.reshape(shape), norm="ortho")  # F^H e_k
        Bf = O.sense_normal_toeplitz(fk, sm, T) + lam * fk
        d_brute[k] = np.fft.fftn(Bf, norm="ortho").ravel()[k].real  # (F B F^H)[k, k]
    P = O.circulant_precond(c, sm, lam)
    assert np.allclose(1.0 / P.ravel(), d_brute, rtol=1e-10, atol=1e-12)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    y = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    assert abs(O.vdot(y, O.precond_apply(P, x)) - O.vdot(O.precond_apply(P, y), x)) < 1e-12
    assert O.vdot(x, O.precond_apply(P, x)).real > 0


def test_torch_fp64_restatement_matches_numpy(golden):
    """The complex128 torch restatement (used for the 128^3 GPU parity tests) equals the
    numpy oracle: on the reference's dense-builder golden case, on a seeded SENSE case with a
    coil subset, and through 6 CG iterations."""
    import torch

    x = golden["x_rnd"]
    nf = int(golden["nf_rnd"])
    c = golden["coords"][:, :nf].astype(np.float64)
    T = O.toeplitz_diagonal(c, x.shape)
    got = O.toeplitz_apply_t(torch.from_numpy(x), torch.from_numpy(T)) * np.prod(O.grid2(x.shape))
    assert O.rel_l2(got, golden["y_rnd"]) < 1e-12

    rng = np.random.default_rng(5)
    N = (8, 6, 10)
    T = O.toeplitz_diagonal(rng.uniform(-np.pi, np.pi, (3, 300)), N)
    sm = rng.standard_normal((4,) + N) + 1j * rng.standard_normal((4,) + N)
    xs = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    coils = [3, 1, 2]
    a = O.sense_normal_toeplitz(xs, sm, T, coils)
    b = O.sense_normal_toeplitz_t(torch.from_numpy(xs), torch.from_numpy(sm), torch.from_numpy(T), coils)
    assert O.rel_l2(b, a) < 1e-13
    lam = 1e-2
    An = O.regularized(lambda v: O.sense_normal_toeplitz(v, sm, T, coils), lam)
    Tt, st = torch.from_numpy(T), torch.from_numpy(sm)
    At = O.regularized(lambda v: O.sense_normal_toeplitz_t(v, st, Tt, coils), lam)
    xn, nn = O.conjugate_gradient(An, a, iters=6)
    xt, nt = O.conjugate_gradient(At, torch.from_numpy(a), iters=6)
    assert nn == nt == 6 and O.rel_l2(xt, xn) < 1e-12


def test_lower_dimensional_nudft_matches_a_direct_sum():
    """The oracle's 2-D and 1-D NUDFTs (the reference's lower-dimensional plans) against an
    explicit double loop / single loop."""
    rng = np.random.default_rng(11)
    for shape in [(4, 6), (5,)]:
        d = len(shape)
        x = rng.uniform(-np.pi, np.pi, (d, 7))
        c = rng.standard_normal((2, 7)) + 1j * rng.standard_normal((2, 7))
        f = O.nudft_type1(x, c, shape, +1)
        k = np.stack(np.meshgrid(*[np.arange(n) - n // 2 for n in shape], indexing="ij"), axis=-1)
        want = np.einsum("tj,...j->t...", c, np.exp(1j * np.tensordot(k, x, axes=([-1], [0]))))
        assert np.allclose(f, want, atol=1e-12)
        g = rng.standard_normal((2,) + shape) + 1j * rng.standard_normal((2,) + shape)
        c2 = O.nudft_type2(x, g, -1)
        want2 = g.reshape(2, -1) @ np.exp(-1j * np.tensordot(k, x, axes=([-1], [0]))).reshape(-1, 7)
        assert np.allclose(c2, want2, atol=1e-12)
