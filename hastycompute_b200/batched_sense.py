"""Batched SENSE operators through the NUFFT, with outer/inner batches, coil subsets, coil
randomisation and the k-space manipulators of the reference.

Mirrors ``hastypy.base.sense`` (``python/python/hastypy/base/sense.py:123-330``) over the C++
``hasty::mri::BatchedSense`` family (``lib/mri/batch_sense.cpp:12-486``):

* an *outer batch* is one trajectory (one frame): ``coord_vec[o]`` [3, nfreq_o];
* an *inner batch* is an image sharing that trajectory (e.g. a velocity encoding):
  images are ``[nouter, ninner, nz, ny, nx]``;
* ``coils`` selects coil maps per outer batch (one list for all, or one list per outer
  batch); ``set_coil_randomization(True, n)`` draws n distinct coils per outer batch
  at each apply, as ``get_coils`` does in the reference;
* the manipulators ``"kdata"``, ``"weighted"``, ``"weighted_kdata"`` of
  ``BatchedSenseNormal`` (``standard_*_manipulator``, ``batch_sense.cpp:452-486``) act
  in k-space between the forward and adjoint NUFFT: ``(F S x - y) * w``.

The reference keeps the data on the host and streams every inner batch through per-device
contexts (``batch_sense.cpp:47-79, 349-450``); here the plans, coil maps, k-space data and
weights stay resident on the device and every apply is a sequence of sm_100a launches.
"""
from __future__ import annotations

import numpy as np
import torch

from .nufft import NufftPlan
from .toeplitz import _check_c64

MANIPULATORS = (None, "kdata", "weighted", "weighted_kdata")


class _BatchedSenseBase:
    def __init__(self, coord_vec, smaps, kdata_vec=None, weights_vec=None, coils=None, ninner_batches=1, tol=1e-5,
                 maxbatch=8):
        if smaps.dim() != 4 or smaps.dtype != torch.complex64 or smaps.device.type != "cuda":
            raise RuntimeError("smaps must be complex64 [ncoils, nz, ny, nx] on a CUDA device")
        self.device = smaps.device
        self.smaps = smaps.contiguous()
        self.ncoils = smaps.shape[0]
        self.dimensions = tuple(smaps.shape[1:])
        self.nouter_batches = len(coord_vec)
        self.ninner_batches = int(ninner_batches)
        self.coils = coils
        self.plans = [NufftPlan(c.to(self.device, torch.float32).contiguous(), self.dimensions, tol=tol,
                                maxbatch=min(maxbatch, self.ncoils)) for c in coord_vec]
        self.nfreqs = [p.nfreq for p in self.plans]
        self.kdata_vec = None if kdata_vec is None else [k.to(self.device).contiguous() for k in kdata_vec]
        self.weights_vec = None if weights_vec is None else \
            [w.to(self.device, torch.float32).reshape(-1).contiguous() for w in weights_vec]
        self.set_coil_randomization()

    def reinit(self, ninner_batches=1, coils=None):
        self.ninner_batches = int(ninner_batches)
        self.coils = coils

    def set_coil_randomization(self, randomize=False, num_rand_coils=16):
        self.randomize_coils = bool(randomize)
        self.num_rand_coils = int(num_rand_coils)

    def get_coils(self):
        """Per outer batch, the coil list of this apply (random draws when randomised)."""
        if self.randomize_coils:
            return [np.random.permutation(self.ncoils)[:self.num_rand_coils].tolist()
                    for _ in range(self.nouter_batches)]
        if self.coils is None:
            return [list(range(self.ncoils))] * self.nouter_batches
        if len(self.coils) and isinstance(self.coils[0], (list, tuple)):
            return [list(c) for c in self.coils]
        return [list(self.coils)] * self.nouter_batches

    def _check_image(self, x, name):
        if tuple(x.shape) != (self.nouter_batches, self.ninner_batches) + self.dimensions:
            raise RuntimeError(f"{name} must be [nouter, ninner, nz, ny, nx] = "
                               f"{(self.nouter_batches, self.ninner_batches) + self.dimensions}")
        _check_c64(x, name, self.device)

    def close(self):
        for p in self.plans:
            p.close()


class BatchedSense(_BatchedSenseBase):
    """Forward: x [nouter, ninner, *dims] -> list over outer batches of [ninner, ncoils, nfreq_o]
    (rows of unselected coils are left zero)."""

    def apply(self, x, out=None):
        self._check_image(x, "input")
        coils = self.get_coils()
        if out is None:
            out = [torch.zeros((self.ninner_batches, self.ncoils, nf), dtype=torch.complex64, device=self.device)
                   for nf in self.nfreqs]
        for o, plan in enumerate(self.plans):
            cl = coils[o]
            for i in range(self.ninner_batches):
                k = plan.sense_forward(x[o, i], self.smaps, cl)
                out[o][i, cl] = k
        return out


class BatchedSenseAdjoint(_BatchedSenseBase):
    """Adjoint: list over outer batches of [ninner, ncoils, nfreq_o] -> [nouter, ninner, *dims]."""

    def apply(self, kin, out=None):
        coils = self.get_coils()
        if out is None:
            out = torch.empty((self.nouter_batches, self.ninner_batches) + self.dimensions, dtype=torch.complex64,
                              device=self.device)
        for o, plan in enumerate(self.plans):
            cl = coils[o]
            idx = torch.tensor(cl, dtype=torch.long, device=self.device)
            for i in range(self.ninner_batches):
                plan.sense_adjoint(kin[o][i].index_select(0, idx).contiguous(), self.smaps, cl, out=out[o, i])
        return out


class BatchedSenseNormal(_BatchedSenseBase):
    """Normal: x [nouter, ninner, *dims] -> sum_c S_c^H F^H m(F S_c x), m the selected manipulator
    (None: identity; "kdata": minus kdata_vec[o][i]; "weighted": times weights_vec[o];
    "weighted_kdata": both)."""

    def apply(self, x, out=None, manipulator=None):
        if manipulator not in MANIPULATORS:
            raise RuntimeError(f"unknown manipulator {manipulator!r}")
        use_k = manipulator in ("kdata", "weighted_kdata")
        use_w = manipulator in ("weighted", "weighted_kdata")
        if use_k and self.kdata_vec is None:
            raise RuntimeError("the kdata manipulators need kdata_vec")
        if use_w and self.weights_vec is None:
            raise RuntimeError("the weighted manipulators need weights_vec")
        self._check_image(x, "input")
        coils = self.get_coils()
        if out is None:
            out = torch.empty_like(x)
        for o, plan in enumerate(self.plans):
            for i in range(self.ninner_batches):
                plan.sense_normal(x[o, i], self.smaps, coils[o],
                                  kdata=self.kdata_vec[o][i] if use_k else None,
                                  weights=self.weights_vec[o] if use_w else None, out=out[o, i])
        return out
