"""SENSE reconstruction from k-space around the Toeplitz normal operator, on the device.

Mirrors the reference's reconstruction driver ``python/python/hastypy/reconstruct_util.py``:

* ``diagonals_and_rhs`` -- ``load_simulated_diag_rhs`` (``:23-95``): per outer batch (a
  trajectory, e.g. one encoding or one frame) the Toeplitz diagonal of its samples
  (optionally density-compensation weighted) and the right-hand side
  ``b = sum_c conj(S_c) F^H (w * y_c)``;
* ``reconstruct_cg_full`` -- ``:478-508`` with ``ToeplitzSenseLinop`` (``:410-434``) and
  ``PrecondLinop`` (``:436-466``): the initial image is scaled by <x, b> / <x, A x>, then
  CG (optionally preconditioned) solves A x = b for every outer batch at once.

Scaling: with F the type-2 NUFFT (isign -1) and F^H the type-1 (isign +1), the explicit
normal operator F^H W F equals 8 prod(N) times this library's Toeplitz operator built from
the same samples and weights, so the right-hand side is divided by 8 prod(N) and
``sum_c S_c^H Top_w S_c x = b`` is exactly the normal equation of the weighted least-squares
problem ||W^(1/2) (F S x - y)||^2.  (The reference mixes torchkbnufft kernels with its own
NUFFT scaling; that constant is not reproduced.)
"""
from __future__ import annotations

import numpy as np
import torch

from .nufft import NufftPlan
from .toeplitz import System, ToeplitzPlan, _check_c64


def diagonals_and_rhs(plan: ToeplitzPlan, coord_vec, kdata_vec, smaps, weights_vec=None, coils=None, tol=1e-6,
                      maxbatch=8):
    """Packed diagonals [nouter, packed] and right-hand sides [nouter, nz, ny, nx].

    coord_vec[o]: float32 [3, nfreq_o]; kdata_vec[o]: complex64 [ncoils, nfreq_o] (coil rows
    in map order); weights_vec[o]: optional float32 [nfreq_o]."""
    _check_c64(smaps, "smaps", plan.device, plan.shape)
    coils = list(range(smaps.shape[0])) if coils is None else [int(c) for c in coils]
    nouter = len(coord_vec)
    packed = torch.empty((nouter, plan.packed_numel()), dtype=torch.float32, device=plan.device)
    rhs = torch.empty((nouter,) + plan.shape, dtype=torch.complex64, device=plan.device)
    scale = 1.0 / (8.0 * float(np.prod(plan.shape)))
    for o in range(nouter):
        coords = coord_vec[o].to(plan.device, torch.float32).contiguous()
        w = None if weights_vec is None else weights_vec[o].to(plan.device, torch.float32).reshape(-1).contiguous()
        packed[o] = plan.build_diagonal(coords, method="nufft", tol=tol, weights=w)
        nplan = NufftPlan(coords, plan.shape, tol=tol, maxbatch=min(maxbatch, len(coils)))
        kd = kdata_vec[o].to(plan.device).reshape(-1, coords.shape[1])
        kd = kd.index_select(0, torch.tensor(coils, device=plan.device)).contiguous()
        nplan.sense_adjoint(kd, smaps, coils, out=rhs[o], weights=w)
        rhs[o] *= scale
        nplan.close()
    return packed, rhs


def reconstruct_cg_full(plan: ToeplitzPlan, packed, rhs, smaps, precond=None, iters=50, lam=0.0, images=None,
                        coils=None, tol=0.0):
    """CG on sum_c S_c^H Top_o S_c + lam I for every outer batch o (reconstruct_util.py:478-508).

    packed [nouter, packed]; rhs [nouter, nz, ny, nx]; precond: optional list of nouter
    preconditioners (``ToeplitzPlan.build_preconditioner``); images: optional initial
    guesses, scaled by <x, b> / <x, A x> first as the reference does.  Returns the images
    [nouter, nz, ny, nx] and the per-system iteration counts."""
    nouter = rhs.shape[0]
    if images is None:
        images = torch.zeros_like(rhs)
    else:
        images = images.reshape(rhs.shape).clone()
        ax = torch.empty_like(images)
        plan.sense_normal(images, ax, smaps, packed, coils=coils, diag_index=list(range(nouter)), lam=lam)
        num = torch.sum(images.conj() * rhs)
        den = torch.sum(images.conj() * ax)
        s = (num / den) if abs(complex(den)) > 0 else torch.tensor(1.0 + 0j)
        s = complex(s)
        if not np.isfinite(s.real):
            s = complex(1.0, s.imag)
        if not np.isfinite(s.imag):
            s = complex(s.real, 0.0)
        images *= s
    systems = [System(images[o], smaps, packed[o], b=rhs[o], coils=coils, lam=lam,
                      precond=None if precond is None else precond[o]) for o in range(nouter)]
    status, done = plan.cg_systems(systems, iters=iters, tol=tol)
    return images, done
