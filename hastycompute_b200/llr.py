"""Locally-low-rank regularisation: block singular-value thresholding and ADMM around the
batched Toeplitz CG, over the C ABI.

Mirrors the reference's

* ``Random3DBlocksSVT`` / ``Normal3DBlocksSVT`` (``lib/op/svt.cpp:268-490``,
  ``python/python/hastypy/base/svt.py:28-61``): x is [d0, d1, S0, S1, S2] (d0 the low-rank
  axis, e.g. frames; d1 e.g. velocity encodings), thresholded in place block by block;
* the scaled ADMM of ``BatchedSenseAdmmConjugateGradientLoader`` / ``Admm::run``
  (``lib/mri/batch_sense.ixx:302-431``, ``lib/op/opalgs.cpp:103-111``): x-update by CG on
  (A^H A + rho/2 I) x = A^H y + rho/2 (z - u), z = SVT(x + u), u += x - z.

The reference runs the blocks of one call concurrently on a thread pool, overlapping
ones included; here blocks are grouped into waves of non-overlapping blocks (one launch
each), applied in order, which makes the result deterministic.  Block shifts and random
corners come from a numpy Generator (``seed``) instead of ``std::default_random_engine``.
"""
from __future__ import annotations

import numpy as np
import torch

from . import capi
from .toeplitz import _check_c64, _ptr, _stream_ptr


def waves_of(corners, block_shape, space_shape=None):
    """Greedy partition of block corners into lists of non-overlapping blocks, keeping the
    input order within and across waves; one voxel-occupancy grid per wave."""
    cs = [tuple(int(v) for v in c) for c in corners]
    if not cs:
        return []
    b = tuple(int(v) for v in block_shape)
    if space_shape is None:
        space_shape = tuple(max(c[d] for c in cs) + b[d] for d in range(3))
    waves, occ = [], []
    for c in cs:
        sl = tuple(slice(c[d], c[d] + b[d]) for d in range(3))
        for w, o in zip(waves, occ):
            if not o[sl].any():
                w.append(c)
                o[sl] = True
                break
        else:
            o = np.zeros(space_shape, bool)
            o[sl] = True
            waves.append([c])
            occ.append(o)
    return waves


def svt_blocks(x, corners, block_shape, thresh, soft=True):
    """Threshold the singular values of the given non-overlapping blocks of x in place."""
    if x.dim() != 5:
        raise RuntimeError("x must be [d0, d1, S0, S1, S2]")
    _check_c64(x, "x", x.device)
    d0, d1, S0, S1, S2 = (int(v) for v in x.shape)
    b0, b1, b2 = (int(v) for v in block_shape)
    cs = np.asarray(corners, dtype=np.int64).reshape(-1, 3)
    if len(cs) == 0:
        return x
    if np.any(cs < 0) or np.any(cs + np.array([b0, b1, b2]) > np.array([S0, S1, S2])):
        raise RuntimeError("a block does not fit inside the image")
    ct = torch.from_numpy(cs.astype(np.int32)).to(x.device)
    capi.check(capi.load().hb_svt_blocks(_ptr(x), d0, d1, S0, S1, S2, b0, b1, b2, _ptr(ct), len(cs), float(thresh),
                                         1 if soft else 0, _stream_ptr(x.device)))
    return x


class _BlocksSVT:
    def __init__(self, input_shape, block_shape, thresh, soft, seed):
        self.input_shape = tuple(int(v) for v in input_shape)
        self.block_shape = tuple(int(v) for v in block_shape)
        self.thresh = float(thresh)
        self.soft = bool(soft)
        self.rng = np.random.default_rng(seed)
        self.last_waves = []

    def update_thresh(self, thresh):
        self.thresh = float(thresh)

    def _run(self, x, waves):
        self.last_waves = waves
        for w in waves:
            svt_blocks(x, w, self.block_shape, self.thresh, self.soft)
        return x


class Random3DBlocksSVT(_BlocksSVT):
    """``nblocks`` blocks at random corners (``Random3DBlocksSVT::apply``, svt.cpp:268-305)."""

    def __init__(self, input_shape, nblocks, block_shape, thresh, soft=True, seed=None):
        super().__init__(input_shape, block_shape, thresh, soft, seed)
        self.nblocks = int(nblocks)

    def apply(self, x):
        bounds = [s - b for s, b in zip(self.input_shape[2:], self.block_shape)]
        corners = [tuple(int(self.rng.integers(0, bd + 1)) for bd in bounds) for _ in range(self.nblocks)]
        return self._run(x, waves_of(corners, self.block_shape, self.input_shape[2:]))


class Normal3DBlocksSVT(_BlocksSVT):
    """A grid of blocks with strides, repeated ``block_iter`` times with random shifts (the
    first unshifted); a block reaching the last index of an axis is skipped, as in
    ``OldNormal3DBlocksSVT::apply`` (svt.cpp:352-440)."""

    def __init__(self, input_shape, block_strides, block_shape, block_iter, thresh, soft=True, seed=None):
        super().__init__(input_shape, block_shape, thresh, soft, seed)
        self.block_strides = tuple(int(v) for v in block_strides)
        if block_iter < 1:
            raise RuntimeError("Can't perform Normal3DBlocksSVT with block_iter < 1")
        self.block_iter = int(block_iter)

    def corners(self):
        S = self.input_shape[2:]
        shifts = [[0] + [int(self.rng.integers(0, b + 1)) for _ in range(self.block_iter - 1)] for b in self.block_shape]
        out = []
        for it in range(self.block_iter):
            sh = [shifts[d][it] for d in range(3)]
            cs = []
            for n0 in range(S[0] // self.block_strides[0]):
                s0 = n0 * self.block_strides[0] + sh[0]
                if s0 + self.block_shape[0] >= S[0]:
                    continue
                for n1 in range(S[1] // self.block_strides[1]):
                    s1 = n1 * self.block_strides[1] + sh[1]
                    if s1 + self.block_shape[1] >= S[1]:
                        continue
                    for n2 in range(S[2] // self.block_strides[2]):
                        s2 = n2 * self.block_strides[2] + sh[2]
                        if s2 + self.block_shape[2] >= S[2]:
                            continue
                        cs.append((s0, s1, s2))
            out.append(cs)
        return out

    def apply(self, x):
        waves = []
        disjoint = all(st >= b for st, b in zip(self.block_strides, self.block_shape))
        for cs in self.corners():  # iterations in order; overlapping blocks of one iteration split into waves
            if disjoint:
                waves.append(cs)
            else:
                waves.extend(waves_of(cs, self.block_shape, self.input_shape[2:]))
        return self._run(x, [w for w in waves if w])


def admm_vectors(stage, x, z, u, b0=None, b=None, rho=1.0):
    n = x.numel()
    capi.check(capi.load().hb_admm_vectors(n, int(stage), _ptr(x), _ptr(z), _ptr(u), _ptr(b0), _ptr(b), float(rho),
                                           _stream_ptr(x.device)))


def admm_llr(plan, x, b0, smaps, packed, rho, svt_op, admm_iters=10, cg_iters=5, coils=None, diag_index=None,
             precond=None):
    """Scaled ADMM with a locally-low-rank prior (``batch_sense.ixx:302-431``): x, b0 are
    [d0, d1, nz, ny, nx] (b0 = A^H y); system (f, e) uses diagonal ``diag_index[f*d1 + e]``
    (default: frame f).  Each x-update is one batched CG over all d0*d1 systems with
    lambda = rho/2 (``precond``: optional per-frame preconditioners, a list of d0 tensors).
    Returns (x, z)."""
    from .toeplitz import System

    d0, d1 = x.shape[:2]
    x4 = x.reshape((d0 * d1,) + plan.shape)
    z = x.clone()
    u = torch.zeros_like(x)
    b = torch.empty_like(x)
    b4 = b.reshape(x4.shape)
    if diag_index is None:
        diag_index = [s // d1 for s in range(d0 * d1)]
    pk = plan.packed_numel()
    packed2 = packed.reshape(-1, pk)
    for _ in range(admm_iters):
        admm_vectors(0, x, z, u, b0, b, rho)
        systems = [System(x4[s], smaps, packed2[diag_index[s]], b=b4[s], coils=coils, lam=0.5 * rho,
                          precond=None if precond is None else precond[s // d1]) for s in range(d0 * d1)]
        plan.cg_systems(systems, iters=cg_iters)
        admm_vectors(1, x, z, u)
        svt_op.apply(z)
        admm_vectors(2, x, z, u)
    return x, z
