"""The reference's LibTorch CPU path for the Toeplitz SENSE normal operator and CG,
restated call for call with the same ATen operators (complex64, FP32).

TEST AND CPU-BASELINE INFRASTRUCTURE ONLY: used by ``tests/`` and by the CPU-baseline and
``--impl reference`` legs of ``bench.py``; never by the product path.

The reference cannot be compiled here (C++20 header units, MSVC/clang-cl presets,
cufinufft/finufft/SymEngine/HighFive absent), so this module replays its calls:
* ``CUDANormalNufftToeplitz::apply_addcmul`` (``lib/fft/nufft.cpp:1181-1188``):
  ``at::fft_fftn_out(s1, in, s=2N, dims)``, ``s1.mul_(diagonal)``,
  ``at::fft_ifftn_out(s2, s1, dims)``, ``add_to.addcmul_(s2.index(0:N), mul)``;
  constructed from a precomputed diagonal (``nufft.cpp:1133-1161``), which is how the
  reference runs on LibTorch-CPU tensors.
* the SENSE coil loop (``lib/mri/sense.ixx:533-577``): ``out.zero_()``, per coil
  ``imstore = x * S_c`` then the Toeplitz ``apply_addcmul(imstore, out, conj(S_c))``.
* ``ConjugateGradient::run`` (``lib/op/opalgs.cpp:50-96``) with ``A + lambda I``:
  ``at::vdot`` in complex64 and ``.item<double>()`` for the scalars.
"""
from __future__ import annotations

import torch


class ToeplitzSenseNormalCPU:
    def __init__(self, diagonal, smaps, coils=None, lam=0.0):
        self.T = diagonal.to(torch.complex64).reshape((1,) + tuple(diagonal.shape[-3:]))
        self.smaps = smaps.to(torch.complex64)
        self.coils = list(range(smaps.shape[0])) if coils is None else list(coils)
        self.lam = float(lam)
        self.N = tuple(smaps.shape[-3:])
        self.M = tuple(self.T.shape[-3:])
        # storage on the diagonal's device: on a CUDA device the same calls are the
        # reference's own GPU path (cuFFT through at::fft_fftn_out, ATen elementwise kernels)
        dev = self.T.device
        self.smaps = self.smaps.to(dev)
        self.s1 = torch.empty((1,) + self.M, dtype=torch.complex64, device=dev)
        self.s2 = torch.empty((1,) + self.M, dtype=torch.complex64, device=dev)
        self.imstore = torch.empty((1,) + self.N, dtype=torch.complex64, device=dev)

    def apply_addcmul(self, inp, add_to, mul):
        torch.fft.fftn(inp, s=self.M, dim=(1, 2, 3), out=self.s1)
        self.s1.mul_(self.T)
        torch.fft.ifftn(self.s1, dim=(1, 2, 3), out=self.s2)
        n0, n1, n2 = self.N
        add_to.addcmul_(self.s2[:, :n0, :n1, :n2], mul)

    def __call__(self, x):
        x = x.reshape((1,) + self.N)
        out = torch.zeros_like(x)
        for c in self.coils:
            torch.mul(x, self.smaps[c], out=self.imstore)
            self.apply_addcmul(self.imstore, out, self.smaps[c].conj())
        if self.lam != 0.0:
            out.add_(x, alpha=self.lam)
        return out


def conjugate_gradient(A, b, x, iters=30, tol=0.0):
    """opalgs.cpp:50-96 on complex64 torch CPU tensors; x is updated in place.
    Returns the number of applies of A performed."""
    napply = 0
    if iters < 1:
        return napply
    r = b - A(x)
    napply += 1
    z = r
    p = z.clone()
    rzold = torch.real(torch.vdot(r.flatten(), z.flatten()))
    resid = float(rzold.item()) ** 0.5
    for _ in range(iters):
        if resid < tol:
            return napply
        Ap = A(p)
        napply += 1
        pAp = torch.real(torch.vdot(p.flatten(), Ap.flatten()))
        if pAp.item() <= 0.0:
            raise RuntimeError("A was not positive definite")
        alpha = rzold / pAp
        x += p * alpha
        r -= Ap * alpha
        z = r
        rznew = torch.real(torch.vdot(r.flatten(), z.flatten()))
        p *= rznew / rzold
        p += z
        rzold = rznew
        resid = float(rzold.item()) ** 0.5
    return napply
