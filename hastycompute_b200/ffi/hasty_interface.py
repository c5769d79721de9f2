"""Thin Python class over torch.classes.HastyInterface.FunctionLambda, with the name and
signature of the reference's hastypy/ffi/hasty_interface.py: a TorchScript function compiled
from source, called as entry(inout, captures), e.g. as NufftNormal's k-space step.

    def apply(a: List[Tensor], b: List[Tensor]):
        for i in range(len(b)):
            a[i] += b[i]
"""
import torch

import hastycompute_b200 as _hc

_hc.load_torch_library()
_mod = torch.classes.HastyInterface


class FunctionLambda:
    def __init__(self, script: str, entry: str, captures: list[torch.Tensor]):
        self._funclam = _mod.FunctionLambda(script, entry, captures)

    def apply(self, input: list[torch.Tensor]):
        self._funclam.apply(input)
