"""The arithmetic of the reduced-precision plan's x pass, emulated on the CPU: the
zero-padded 2nx-point DFT of nx = 128 samples as a contraction of BF16 hi + lo operands with
FP32-or-better accumulation.  Keeping the three products hi*hi + hi*lo + lo*hi meets the
reduced-precision bar (1e-4) with two orders of magnitude to spare; dropping either cross
product does not, which is why the tensor-core pass issues three contractions per real
product."""
import numpy as np


def _bf16(a):
    """Round float32 values to BF16 (nearest, ties to even), returned as float64."""
    u = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def _split(a):
    hi = _bf16(a)
    lo = _bf16(np.asarray(a, np.float32) - hi.astype(np.float32))
    return hi, lo


def _contraction_error(products):
    rng = np.random.default_rng(0)
    nx, m = 128, 256
    a = (rng.standard_normal((64, nx)) + 1j * rng.standard_normal((64, nx))).astype(np.complex64)
    kx, x = np.arange(m)[:, None], np.arange(nx)[None, :]
    f = np.exp(-2j * np.pi * ((kx * x) % m) / m)
    exact = a.astype(np.complex128) @ f.T
    ar, ai, fr, fi = _split(a.real), _split(a.imag), _split(f.real), _split(f.imag)

    def real_product(u, v):  # sum of the kept hi/lo products of u @ v.T
        return sum(u[i] @ v[j].T for i, j in products)

    re = real_product(ar, fr) - real_product(ai, fi)
    im = real_product(ar, fi) + real_product(ai, fr)
    return np.linalg.norm(re + 1j * im - exact) / np.linalg.norm(exact)


def test_three_products_meet_the_bar():
    assert _contraction_error([(0, 0), (0, 1), (1, 0)]) < 1e-5  # 3.8e-6


def test_dropping_a_cross_product_fails_the_bar():
    assert _contraction_error([(0, 0), (0, 1)]) > 1e-4  # no lo part of the samples: 1.7e-3
    assert _contraction_error([(0, 0), (1, 0)]) > 1e-4  # no lo part of the DFT rows: 1.3e-3
    assert _contraction_error([(0, 0)]) > 1e-4
