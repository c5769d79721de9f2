"""Location of the native libraries (counterpart of hastypy/ffi/hasty_ffi.py:8-22)."""
import os

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def get_ffi_libfile():
    """The TorchScript library with the HastyToeplitz, HastyNufft and HastySVT classes."""
    return os.path.join(_PKG, "libhasty_torch.so")


def get_capi_libfile():
    """The C-ABI library with the CUDA kernels."""
    return os.path.join(_PKG, "libhasty_b200.so")
