"""B200-native Toeplitz-embedded SENSE normal operator and batched CG (sm_100a).

Native pieces (built in-tree by ``hastycompute_b200.build``):
  libhasty_b200.so  CUDA kernels + C ABI (include/hasty_b200.h)
  libhasty_torch.so C++/LibTorch host layer and TorchScript classes
"""
from . import capi  # noqa: F401

__version__ = "0.1.0"


def load_torch_library():
    """Load the TorchScript classes (torch.classes.HastyToeplitz*)."""
    import os

    import torch

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libhasty_torch.so")
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing; build it with `python -m hastycompute_b200.build`")
    capi.load()
    torch.classes.load_library(path)
    return path
