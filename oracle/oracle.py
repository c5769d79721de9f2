"""FP64 CPU oracle for the Toeplitz-embedded SENSE normal operator and its CG solver.

TEST INFRASTRUCTURE ONLY.  This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import it.
The product path (``hastycompute_b200``) never calls it.

It restates, in numpy float64, the reference algorithm (HastyCompute, C++ over
LibTorch).  File references below are paths inside the reference project:

* ``lib/fft/nufft.cpp:932-971``   ``build_diagonal_base``: a unit impulse at index
  M/2 of the 2x grid, NUFFT type-2 (isign -1) then type-1 (isign +1), each scaled
  by ``1/sqrt(prod(M))`` (``nufft.cpp:104-123``), then ``ifftshift`` and ``fftn``.
  A type-2 NUFFT of a centred impulse is a constant, so the construction equals the
  direct NUDFT  ``psf(d) = prod(M)^-1 * sum_j exp(+i c_j . d)``  for d in [-N, N)^3,
  stored circulantly (index n <-> d = n for n < M/2, d = n - M otherwise).
  Here it is evaluated exactly (float64, no NUFFT tolerance).
* ``lib/fft/nufft.cpp:1163-1197``  ``apply``/``apply_add``/``apply_addcmul``/
  ``apply_inplace``: ``y = ifftn(T * fftn(x, s=M))[:N0, :N1, :N2]`` (high-end zero
  pad, inverse scaled by 1/prod(M)).
* ``lib/mri/sense.ixx:500-578``  ``sense_normal_apply`` with the Toeplitz body
  (``apply_addcmul(x*S_c, out, conj(S_c))``): ``out = sum_c conj(S_c) * Top(S_c * x)``.
* ``lib/op/opalgs.cpp:50-96``  ``ConjugateGradient::run`` (r = b - A x, p = z, the
  tol test on sqrt(rz), the positive-definiteness check) applied to ``A + lambda*I``
  (``python/python/hastypy/base/torch_opalg.py:49-61``).
* ``lib/fft/nufft.cpp:540-767`` the type-1 / type-2 NUFFTs of ``CUDANufft`` and the SENSE
  forward / adjoint around them (``lib/mri/sense.ixx:426-497``), as direct NUDFTs.
* ``lib/mri/precond.cpp:65-117`` the circulant preconditioner (the Fourier-domain diagonal of
  the SENSE normal operator, inverted) and its apply.
* ``lib/op/svt.cpp:11-490`` block singular-value thresholding (locally low rank) and the
  scaled ADMM around CG (``lib/op/opalgs.cpp:103-111``, ``lib/mri/batch_sense.ixx:302-431``).
* ``lib/fft/nufft.cpp:410-767`` / ``:785-920`` explicit NUFFT normal op on the N grid
  (type-2 then type-1, each /sqrt(prod(N))), evaluated as a dense direct NUDFT.
  ``Toeplitz = explicit / 2^3`` in 3D because of the two different grid scalings.

Coordinate convention (``nufft.cpp:192-197``, ``:578-585``): ``coords`` is [3, K];
row a pairs with image axis a (z, y, x order, x fastest in memory).
"""
from __future__ import annotations

import numpy as np


def grid2(nmodes):
    """The Toeplitz embedding grid: every spatial axis doubled (``nufft.cpp:978-981``)."""
    return tuple(2 * int(n) for n in nmodes)


def _axis_phasors(c, d):
    """exp(+i * c_j * d) for a coordinate row c [K] and integer offsets d [L] -> [K, L]."""
    return np.exp(1j * np.outer(np.asarray(c, np.float64), np.asarray(d, np.float64)))


def _circ_offsets(m):
    """Signed offset d for every index n of a length-m circulant axis."""
    n = np.arange(m)
    return np.where(n < m // 2, n, n - m)


def psf_circulant(coords, nmodes, weights=None, chunk=4096):
    """PSF on the 2x grid in circulant layout (``nufft.cpp:932-971`` after ifftshift).

    psf[n0,n1,n2] = prod(M)^-1 * sum_j w_j exp(+i (c0_j d0 + c1_j d1 + c2_j d2)).
    """
    coords = np.asarray(coords, np.float64)
    M = grid2(nmodes)
    K = coords.shape[1]
    w = np.ones(K) if weights is None else np.asarray(weights, np.float64)
    out = np.zeros(M, np.complex128)
    d = [_circ_offsets(m) for m in M]
    for s in range(0, K, chunk):
        e = slice(s, min(K, s + chunk))
        pz = _axis_phasors(coords[0, e], d[0]) * w[e, None]
        py = _axis_phasors(coords[1, e], d[1])
        px = _axis_phasors(coords[2, e], d[2])
        pzy = (pz[:, :, None] * py[:, None, :]).reshape(pz.shape[0], -1)
        out += (pzy.T @ px).reshape(M)
    return out / float(np.prod(M))


def toeplitz_diagonal(coords, nmodes, weights=None):
    """T = fftn(psf) on the 2x grid, complex128 [M0, M1, M2] (``nufft.cpp:967-969``)."""
    return np.fft.fftn(psf_circulant(coords, nmodes, weights))


def toeplitz_apply(x, T):
    """``CUDANormalNufftToeplitz::apply`` (``nufft.cpp:1163-1170``): crop(ifftn(T*fftn(pad x)))."""
    x = np.asarray(x, np.complex128)
    N = x.shape
    F = np.fft.fftn(x, s=T.shape, axes=(0, 1, 2))
    y = np.fft.ifftn(F * T)
    return y[: N[0], : N[1], : N[2]]


def sense_normal_toeplitz(x, smaps, T, coils=None):
    """Toeplitz SENSE normal op (``sense.ixx:500-578`` + ``nufft.cpp:1181-1188``).

    out.zero_(); for c in coils: out += conj(S_c) * Top(S_c * x)
    """
    x = np.asarray(x, np.complex128)
    smaps = np.asarray(smaps, np.complex128)
    if coils is None:
        coils = range(smaps.shape[0])
    out = np.zeros_like(x)
    for c in coils:
        out += np.conj(smaps[c]) * toeplitz_apply(x * smaps[c], T)
    return out


# ---- the same two restatements on complex128 torch tensors ----
# At the benchmark's size (128^3 images, 256^3 grid, 16 coils) numpy's FFTs take minutes per
# CG solve.  These restate nufft.cpp:1163-1197 and sense.ixx:500-578 line for line with
# torch.fft in complex128 (FP64), on whichever device the tensors live on; the CG below
# accepts them as well.  tests/test_oracle.py pins them to the numpy versions above.

def toeplitz_apply_t(x, T):
    """``toeplitz_apply`` for complex128 torch tensors: crop(ifftn(T * fftn(x, s=M)))."""
    import torch

    N = tuple(x.shape)
    F = torch.fft.fftn(x.to(torch.complex128), s=tuple(T.shape), dim=(0, 1, 2))
    F.mul_(T)
    y = torch.fft.ifftn(F, dim=(0, 1, 2))
    return y[: N[0], : N[1], : N[2]]


def sense_normal_toeplitz_t(x, smaps, T, coils=None):
    """``sense_normal_toeplitz`` for complex128 torch tensors (x [N], smaps [C, N], T [M])."""
    import torch

    x = x.to(torch.complex128)
    if coils is None:
        coils = range(smaps.shape[0])
    out = torch.zeros_like(x)
    for c in coils:
        s = smaps[c].to(torch.complex128)
        out += s.conj() * toeplitz_apply_t(x * s, T)
    return out


def explicit_normal(x, coords, weights=None):
    """Explicit NUFFT normal op on the N grid (type-2 isign -1, type-1 isign +1, each
    scaled 1/sqrt(prod(N)); ``nufft.cpp:104-123,785-920``), as a dense direct NUDFT."""
    x = np.asarray(x, np.complex128)
    coords = np.asarray(coords, np.float64)
    N = x.shape
    K = coords.shape[1]
    w = np.ones(K) if weights is None else np.asarray(weights, np.float64)
    k = [np.arange(n) - n // 2 for n in N]  # CMCL mode ordering
    ez = _axis_phasors(coords[0], k[0])
    ey = _axis_phasors(coords[1], k[1])
    ex = _axis_phasors(coords[2], k[2])
    # type 2: f_j = sum_k x_k exp(-i k.c_j)
    f = np.einsum("jz,jy,jx,zyx->j", ez.conj(), ey.conj(), ex.conj(), x, optimize=True)
    f = f * w
    # type 1: y_k = sum_j f_j exp(+i k.c_j)
    y = np.einsum("j,jz,jy,jx->zyx", f, ez, ey, ex, optimize=True)
    return y / float(np.prod(N))


_AXES = "zyx"


def nudft_type1(coords, c, nmodes, isign=+1):
    """Direct FP64 type-1 NUDFT, the transform ``hasty::fft::CUDANufft`` type 1 computes
    through cufinufft (``lib/fft/nufft.cpp:640-700``; options ``nufft.ixx:46-48``):
    f[t, k] = sum_j c[t, j] exp(isign * i * k . x_j), centred modes k = i - n//2,
    c [ntransf, K] -> f [ntransf, *nmodes]; d = len(nmodes) = coords.shape[0] in 1..3 (the
    reference's 1-D, 2-D and 3-D plans, ``nufft.ixx:72-160``)."""
    coords = np.asarray(coords, np.float64)
    c = np.atleast_2d(np.asarray(c, np.complex128))
    d = len(nmodes)
    k = [np.arange(n) - n // 2 for n in nmodes]
    e = [np.exp(isign * 1j * np.outer(coords[a], k[a])) for a in range(d)]
    ax = _AXES[3 - d:]
    return np.einsum("tj," + ",".join("j" + a for a in ax) + "->t" + ax, c, *e, optimize=True)


def nudft_type2(coords, f, isign=-1):
    """Direct FP64 type-2 NUDFT (``lib/fft/nufft.cpp:702-767``):
    c[t, j] = sum_k f[t, k] exp(isign * i * k . x_j), f [ntransf, *nmodes] -> c [ntransf, K]
    (d = coords.shape[0] transformed axes, 1..3)."""
    coords = np.asarray(coords, np.float64)
    d = coords.shape[0]
    f = np.asarray(f, np.complex128)
    if f.ndim == d:
        f = f[None]
    k = [np.arange(n) - n // 2 for n in f.shape[1:]]
    e = [np.exp(isign * 1j * np.outer(coords[a], k[a])) for a in range(d)]
    ax = _AXES[3 - d:]
    return np.einsum("t" + ax + "," + ",".join("j" + a for a in ax) + "->tj", f, *e, optimize=True)


def sense_adjoint(coords, kdata, smaps, coils=None):
    """SENSE adjoint with the type-1 NUFFT (``lib/mri/sense.ixx:426-497``):
    out = sum_b conj(S[coils[b]]) * type1(kdata[b])."""
    smaps = np.asarray(smaps, np.complex128)
    coils = range(smaps.shape[0]) if coils is None else coils
    imgs = nudft_type1(coords, kdata, smaps.shape[1:], +1)
    return sum(np.conj(smaps[c]) * imgs[b] for b, c in enumerate(coils))


def sense_forward(coords, x, smaps, coils=None):
    """SENSE forward with the type-2 NUFFT: kdata[b] = type2(S[coils[b]] * x)."""
    smaps = np.asarray(smaps, np.complex128)
    coils = range(smaps.shape[0]) if coils is None else coils
    return nudft_type2(coords, np.stack([smaps[c] * x for c in coils]), -1)


def sense_normal_nufft(coords, x, smaps, coils=None, kdata=None, weights=None):
    """NUFFT SENSE normal operator with the reference's k-space manipulators
    (``lib/mri/batch_sense.cpp:452-486``): sum_b conj(S_cb) type1(w * (type2(S_cb x) - kdata[cb]))."""
    smaps = np.asarray(smaps, np.complex128)
    coils = list(range(smaps.shape[0])) if coils is None else list(coils)
    k = sense_forward(coords, x, smaps, coils)
    if kdata is not None:
        k = k - np.asarray(kdata, np.complex128)[coils]
    if weights is not None:
        k = k * np.asarray(weights, np.float64)[None]
    return sense_adjoint(coords, k, smaps, coils)


def circulant_precond(coords, smaps, lam=0.0, coils=None):
    """Circulant preconditioner (``CirculantPreconditionerOp::build_diagonal``,
    ``lib/mri/precond.cpp:65-117``; ``torch_precond.py:60-105``, both ported from sigpy):
    1 / (d + lam) with d[k] = (F B F^H)[k, k] the Fourier-domain diagonal of
    B = sum_c S_c^H Top S_c, in FFT (uncentred) order, float64:
    d = FFT_2N(psf * IFFT_2N(sum_c |FFT_2N(pad(conj S_c))|^2))[::2, ::2, ::2] / prod(N)."""
    smaps = np.asarray(smaps, np.complex128)
    coils = range(smaps.shape[0]) if coils is None else coils
    N = smaps.shape[1:]
    M = grid2(N)
    psf = psf_circulant(coords, N)
    q = 0.0
    for c in coils:
        q = q + np.abs(np.fft.fftn(np.conj(smaps[c]), s=M, axes=(0, 1, 2))) ** 2
    g = psf * np.fft.ifftn(q)
    d = np.fft.fftn(g)[::2, ::2, ::2].real / float(np.prod(N)) + lam
    return np.where(d > 0, 1.0 / np.where(d > 0, d, 1.0), 1.0)


def precond_apply(P, x):
    """``CirculantPreconditionerOp::apply`` (``precond.cpp:30-52``) in FFT order:
    IFFT(P * FFT(x))."""
    return np.fft.ifftn(P * np.fft.fftn(np.asarray(x, np.complex128)))


def svt_blocks(x, corners, block_shape, thresh, soft=True):
    """Block singular-value thresholding (``lib/op/svt.cpp``): for each corner in order,
    extract the block of x [d0, d1, S0, S1, S2] as the matrix [d1*b0*b1*b2, d0]
    (``extract_block``, ``:11-58``), threshold its singular values (``svt_soft`` /
    ``svt_hard``, ``:60-168``: soft s -> max(s - thresh, 0), hard keeps round(thresh)) and
    insert it back (``insert_block``, ``:170-240``).  float64."""
    y = np.array(x, np.complex128)
    d0, d1 = y.shape[:2]
    b0, b1, b2 = block_shape
    for c0, c1, c2 in corners:
        sl = (slice(None), slice(None), slice(c0, c0 + b0), slice(c1, c1 + b1), slice(c2, c2 + b2))
        M = y[sl].reshape(d0, -1).T
        U, S, Vh = np.linalg.svd(M, full_matrices=False)
        if soft:
            S = np.maximum(S - thresh, 0.0)
        else:
            S[int(thresh + 0.5):] = 0.0
        y[sl] = ((U * S) @ Vh).T.reshape(d0, d1, b0, b1, b2)
    return y


def admm_llr(A_of_system, b0, x0, rho, svt, admm_iters, cg_iters):
    """Scaled ADMM for min ||S x - y||^2 + R(z) s.t. x = z (``lib/op/opalgs.cpp:103-111``,
    ``lib/mri/batch_sense.ixx:302-431``): x-update by CG on (A + rho/2 I) x = b0 + rho/2 (z - u)
    per system (A_of_system(s) is system s's normal operator), z = prox(x + u), u += x - z.
    x0, b0: [d0, d1, *image]; svt(v) returns the proximal step of v."""
    x = np.array(x0, np.complex128)
    z = x.copy()
    u = np.zeros_like(x)
    d0, d1 = x.shape[:2]
    for _ in range(admm_iters):
        b = b0 + 0.5 * rho * (z - u)
        for f in range(d0):
            for e in range(d1):
                A = regularized(A_of_system(f, e), 0.5 * rho)
                x[f, e], _ = conjugate_gradient(A, b[f, e], x0=x[f, e], iters=cg_iters)
        z = svt(x + u)
        u = u + x - z
    return x, z


def _is_torch(a):
    return type(a).__module__.split(".")[0] == "torch"


def vdot(a, b):
    """``vdot`` (``lib/op/vec.cpp:624-637``): sum(conj(a) * b), in FP64."""
    if _is_torch(a):
        import torch

        return complex(torch.vdot(a.flatten(), b.flatten()).item())
    return np.vdot(np.asarray(a).ravel(), np.asarray(b).ravel())


class NotPositiveDefinite(RuntimeError):
    pass


def conjugate_gradient(A, b, x0=None, iters=30, tol=0.0, P=None):
    """``ConjugateGradient::run`` (``lib/op/opalgs.cpp:50-96``), float64.

    Returns (x, n_done) where n_done counts the iterations that updated x.  b (and x0) are
    numpy arrays or torch tensors; either way the vectors are complex128.
    """
    if _is_torch(b):
        import torch

        b = b.to(torch.complex128)
        x = torch.zeros_like(b) if x0 is None else x0.to(torch.complex128).clone()
    else:
        b = np.asarray(b, np.complex128)
        x = np.zeros_like(b) if x0 is None else np.array(x0, np.complex128)
    if iters < 1:
        return x, 0
    r = b - A(x)
    z = P(r) if P is not None else r
    p = z.clone() if _is_torch(z) else z.copy()
    rzold = vdot(r, z).real
    resid = np.sqrt(rzold)
    done = 0
    for _ in range(iters):
        if resid < tol:
            return x, done
        Ap = A(p)
        pAp = vdot(p, Ap).real
        if pAp <= 0.0:
            raise NotPositiveDefinite("A was not positive definite")
        alpha = rzold / pAp
        x = x + alpha * p
        r = r - alpha * Ap
        z = P(r) if P is not None else r
        rznew = vdot(r, z).real
        p = p * (rznew / rzold) + z
        rzold = rznew
        resid = np.sqrt(rzold)
        done += 1
    return x, done


def regularized(A, lam):
    """``A + lambda*I`` (``hastypy/base/torch_opalg.py:49-61``)."""
    return lambda v: A(v) + lam * v


def rel_l2(a, b):
    if _is_torch(a) or _is_torch(b):
        import torch

        dev = a.device if _is_torch(a) else b.device
        a = (a if _is_torch(a) else torch.from_numpy(np.asarray(a))).to(dev, torch.complex128)
        b = (b if _is_torch(b) else torch.from_numpy(np.asarray(b))).to(dev, torch.complex128)
        return float(torch.linalg.vector_norm(a - b) / max(float(torch.linalg.vector_norm(b)), 1e-300))
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
