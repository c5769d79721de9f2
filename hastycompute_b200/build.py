"""Build the in-tree native libraries (sm_100a).

* ``libhasty_b200.so``  -- the CUDA kernels and the C ABI (``include/hasty_b200.h``),
  compiled by nvcc for ``sm_100a`` only.
* ``libhasty_torch.so`` -- the C++20/LibTorch host layer (``hasty::fft``/``mri``/``op``
  classes and the TorchScript custom classes), linked against ``libhasty_b200.so``.

Both land next to this file so they travel with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
CAPI_SO = os.path.join(HERE, "libhasty_b200.so")
TORCH_SO = os.path.join(HERE, "libhasty_torch.so")

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr",
]

CAPI_SOURCES = ["capi.cu", "nufft.cu", "precond.cu", "svt.cu"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps(pattern_dirs, exts):
    files = []
    for d in pattern_dirs:
        for root, _, names in os.walk(d):
            for n in names:
                if os.path.splitext(n)[1] in exts:
                    files.append(os.path.join(root, n))
    return files


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_capi(force=False, verbose=False):
    deps = _deps([CSRC], {".cu", ".cuh", ".h"}) + [os.path.join(ROOT, "include", "hasty_b200.h")]
    deps = [d for d in deps if os.sep + "host" + os.sep not in d]
    if not force and not _stale(CAPI_SO, deps):
        return CAPI_SO
    srcs = [os.path.join(CSRC, s) for s in CAPI_SOURCES]
    tmp = CAPI_SO + ".tmp"
    cmd = [_nvcc()] + NVCC_FLAGS + srcs + ["-o", tmp]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, CAPI_SO)
    return CAPI_SO


def build_torch(force=False, verbose=False):
    """Compile the LibTorch host layer into libhasty_torch.so (needs libhasty_b200.so)."""
    build_capi(force=False, verbose=verbose)
    host = os.path.join(CSRC, "host")
    srcs = sorted(os.path.join(host, f) for f in os.listdir(host) if f.endswith(".cpp"))
    deps = srcs + _deps([host], {".hpp", ".h"}) + [os.path.join(ROOT, "include", "hasty_b200.h"), CAPI_SO]
    if not force and not _stale(TORCH_SO, deps):
        return TORCH_SO
    import torch
    from torch.utils import cpp_extension

    inc = cpp_extension.include_paths() + [os.path.join(ROOT, "include"), host, "/usr/local/cuda/include"]
    libdirs = cpp_extension.library_paths()
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    cmd = ["g++", "-O2", "-std=c++20", "-fPIC", "-shared", f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
           "-DTORCH_API_INCLUDE_EXTENSION_H", "-Wno-deprecated-declarations"]
    for i in inc:
        cmd += ["-I", i]
    cmd += srcs
    for ld in libdirs:
        cmd += ["-L", ld, f"-Wl,-rpath,{ld}"]
    cmd += ["-L", HERE, "-l:libhasty_b200.so", "-Wl,-rpath,$ORIGIN",
            "-lc10", "-ltorch", "-ltorch_cpu", "-ltorch_cuda", "-lc10_cuda",
            "-L/usr/local/cuda/lib64", "-lcudart"]
    tmp = TORCH_SO + ".tmp"
    cmd += ["-o", tmp]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, TORCH_SO)
    return TORCH_SO


def build_all(force=False, verbose=False):
    build_capi(force=force, verbose=verbose)
    if os.path.isdir(os.path.join(CSRC, "host")):
        build_torch(force=force, verbose=verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True)
