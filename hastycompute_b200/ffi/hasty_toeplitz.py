"""Thin Python classes over torch.classes.HastyToeplitz, mirroring the reference's
hastypy/ffi/hasty_sense.py (Sense/SenseNormal/BatchedSenseNormal wrappers).

All tensors are complex64.  Single-system operators take CUDA tensors; the batched
operator accepts CPU or CUDA tensors, like the reference's BatchedSense classes."""
import torch

import hastycompute_b200 as _hc

_hc.load_torch_library()
_mod = torch.classes.HastyToeplitz


class NormalNufftToeplitz:
    """hasty::fft::CUDANormalNufftToeplitz: build from a trajectory (coords [3, K] float32)
    or take a precomputed diagonal [1, 2nz, 2ny, 2nx]."""

    def __init__(self, coords, nmodes, diagonal=None):
        self._op = _mod.NormalNufftToeplitz(coords, list(nmodes), diagonal)

    def apply(self, input, storage1, storage2):
        return self._op.apply(input, storage1, storage2)

    def apply_add(self, input, add_to, storage1, storage2):
        self._op.apply_add(input, add_to, storage1, storage2)

    def apply_addcmul(self, input, add_to, mul, storage1, storage2):
        self._op.apply_addcmul(input, add_to, mul, storage1, storage2)

    def apply_inplace(self, input, storage1, storage2):
        self._op.apply_inplace(input, storage1, storage2)

    def get_diagonal(self):
        return self._op.get_diagonal()

    def set_precision(self, precision):
        """"fp32" (default) or "bf16x3": the forward x pass as a tensor-core contraction with
        BF16 hi + lo operands and FP32 accumulation (ny = nx = 128)."""
        self._op.set_precision(precision)


class SenseNormalToeplitz:
    """Toeplitz twin of hastypy.ffi.hasty_sense.SenseNormal (same apply signature)."""

    def __init__(self, coords, nmodes, diagonal=None):
        self._senseop = _mod.SenseNormalToeplitz(coords, list(nmodes), diagonal)

    def apply(self, input, output, smaps, coils, imspace_storage=None, kspace_storage=None):
        self._senseop.apply(input, output, smaps, list(coils), imspace_storage, kspace_storage)

    def get_diagonal(self):
        return self._senseop.get_diagonal()

    def set_precision(self, precision):
        """"fp32" (default) or "bf16x3": the forward x pass as a tensor-core contraction with
        BF16 hi + lo operands and FP32 accumulation (ny = nx = 128)."""
        self._senseop.set_precision(precision)


class BatchedSenseNormalToeplitz:
    """Toeplitz twin of hastypy.ffi.hasty_sense.BatchedSenseNormal: outer batches are
    systems; diag_index maps each outer batch to one of the diagonals."""

    def __init__(self, diagonals, smaps, diag_index=None):
        self._senseop = _mod.BatchedSenseNormalToeplitz(diagonals, smaps, diag_index)

    def apply(self, input, output, coils=None, lamda=0.0):
        if lamda == 0.0:
            self._senseop.apply(input, output, coils)
        else:
            self._senseop.apply_regularized(input, output, float(lamda), coils)

    def set_precision(self, precision):
        """"fp32" (default) or "bf16x3": the forward x pass as a tensor-core contraction with
        BF16 hi + lo operands and FP32 accumulation (ny = nx = 128)."""
        self._senseop.set_precision(precision)

    def cg(self, x, b, iters=30, tol=0.0, lamda=0.0, coils=None, precond=None, centered=True):
        """ConjugateGradient on (A^H A)_toeplitz + lamda I for every outer batch of x (in
        place).  With ``precond`` (a circulant preconditioner diagonal, centred as
        ``circulant_precond_diagonal`` returns it unless ``centered=False``) the solve is
        preconditioned CG with CirculantPreconditionerOp(precond, centered)."""
        if precond is None:
            return self._senseop.cg(x, b, int(iters), float(tol), float(lamda), coils)
        return self._senseop.pcg(x, b, int(iters), float(tol), float(lamda), coils, precond, bool(centered))


def circulant_precond_diagonal(smaps, coord, lamda=0.0):
    """CirculantPreconditionerOp::build_diagonal (precond.cpp:65-117): the centred inverse
    Fourier-domain diagonal of the SENSE normal operator plus lamda, float32 [nz, ny, nx]."""
    return torch.ops.HastyToeplitz.circulant_precond_diagonal(smaps, coord, float(lamda))


def batched_sense_toeplitz_diagonals(input, coil_list, smaps, diagonals, streams=None):
    """The binding called by the reference's ToeplitzSenseLinop (reconstruct_util.py:410-434)."""
    torch.ops.HastyToeplitz.batched_sense_toeplitz_diagonals(input, coil_list, smaps, diagonals, streams)
