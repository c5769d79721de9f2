"""Thin Python classes over torch.classes.HastyNufft, with the names and signatures of the
reference's hastypy/ffi/hasty_nufft.py (NufftOptions, Nufft, NufftNormal).  Tensors are CUDA
complex64, coordinates CUDA float32 [3, nfreq]."""
import torch

import hastycompute_b200 as _hc

_hc.load_torch_library()
_mod = torch.classes.HastyNufft


class NufftOptions:
    def __init__(self, type: int, positive: bool | None = None, tol: float | None = None):
        self._nufftopts = _mod.NufftOptions(type, positive, tol)

    @staticmethod
    def type2():
        return NufftOptions(2, False, 1e-5)

    @staticmethod
    def type1():
        return NufftOptions(1, True, 1e-5)


class Nufft:
    def __init__(self, coord: torch.Tensor, nmodes: list[int], opts: NufftOptions):
        self._nufftopt = _mod.Nufft(coord, list(nmodes), opts._nufftopts)

    def apply(self, input: torch.Tensor, output: torch.Tensor):
        self._nufftopt.apply(input, output)


class NufftNormal:
    def __init__(self, coord: torch.Tensor, nmodes: list[int], forward_opts: NufftOptions, backward_opts: NufftOptions):
        self._nufftopt = _mod.NufftNormal(coord, list(nmodes), forward_opts._nufftopts, backward_opts._nufftopts)

    def apply(self, input: torch.Tensor, output: torch.Tensor, storage: torch.Tensor, callable=None):
        """output = type1(f(type2(input))) with storage holding the k-space data in between;
        f is `callable` (a FunctionLambda, applied in place) or the identity."""
        self._nufftopt.apply(input, output, storage, callable._funclam if callable is not None else None)
