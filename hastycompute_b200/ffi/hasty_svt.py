"""Thin Python classes over torch.classes.HastySVT, with the names and signatures of the
reference's hastypy/ffi/hasty_svt.py (Random3DBlocksSVT, Normal3DBlocksSVT).  The input is
complex64 [d0, d1, S0, S1, S2] on the CPU or a CUDA device, thresholded in place; `streams`
is accepted for compatibility (the work runs on the current CUDA stream)."""
import torch

import hastycompute_b200 as _hc

_hc.load_torch_library()
_mod = torch.classes.HastySVT


class Random3DBlocksSVT:
    def __init__(self, streams: list[torch.Stream] | None = None):
        self._svtop = _mod.Random3DBlocksSVT(None)

    def apply(self, input: torch.Tensor, nblocks: int, block_shape: list[int], thresh: float, soft: bool):
        self._svtop.apply(input, nblocks, list(block_shape), thresh, soft)


class Normal3DBlocksSVT:
    def __init__(self, streams: list[torch.Stream] | None = None):
        self._svtop = _mod.Normal3DBlocksSVT(None)

    def apply(self, input: torch.Tensor, block_strides: list[int], block_shape: list[int], block_iter: int,
              thresh: float, soft: bool):
        self._svtop.apply(input, list(block_strides), list(block_shape), block_iter, thresh, soft)
