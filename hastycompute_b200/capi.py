"""ctypes binding of the C ABI (``include/hasty_b200.h``) in ``libhasty_b200.so``.

Loading fails loudly when the native library is missing: there is no Python or CPU
fallback for the operator.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libhasty_b200.so")

HB_OK = 0
HB_ERR_INVALID = 1
HB_ERR_UNSUPPORTED = 2
HB_ERR_CUDA = 3
HB_ERR_WORKSPACE = 4
HB_ERR_NOT_PD = 5

HB_NOALLOC_SCRATCH_BYTES = 16 << 20
HB_PRECISION_FP32 = 0
HB_PRECISION_BF16X3 = 1

HB_CG_RUNNING = 0
HB_CG_CONVERGED = 1
HB_CG_NOT_PD = 2

c_void_p = ctypes.c_void_p
c_int = ctypes.c_int
c_i64 = ctypes.c_int64
c_size = ctypes.c_size_t
c_float = ctypes.c_float
c_double = ctypes.c_double
P_i64 = ctypes.POINTER(ctypes.c_int64)
P_i32 = ctypes.POINTER(ctypes.c_int32)

HB_CG_GRAPH = 1


class HbSystem(ctypes.Structure):
    """struct hb_system (include/hasty_b200.h)."""
    _fields_ = [("x", ctypes.c_void_p), ("out", ctypes.c_void_p), ("b", ctypes.c_void_p),
                ("smaps", ctypes.c_void_p), ("coils", ctypes.POINTER(ctypes.c_int64)), ("ncoil", ctypes.c_int64),
                ("packed_diag", ctypes.c_void_p), ("lam", ctypes.c_float), ("precond", ctypes.c_void_p)]


P_sys = ctypes.POINTER(HbSystem)

# name -> (restype, argtypes); one entry per declaration of include/hasty_b200.h
SIGNATURES = {
    "hb_version": (c_int, []),
    "hb_last_error": (ctypes.c_char_p, []),
    "hb_size_supported": (c_int, [c_i64, c_i64, c_i64]),
    "hb_plan_create": (c_int, [ctypes.POINTER(c_void_p), c_i64, c_i64, c_i64, c_int]),
    "hb_plan_destroy": (c_int, [c_void_p]),
    "hb_plan_set_precision": (c_int, [c_void_p, c_int]),
    "hb_plan_precision": (c_int, [c_void_p]),
    "hb_wait_status": (c_int, [c_int]),
    "hb_plan_inject_tc_stall": (c_int, [c_void_p, c_int]),
    "hb_plan_inject_x_stall": (c_int, [c_void_p, c_int]),
    "hb_diag_packed_floats": (c_i64, [c_void_p]),
    "hb_diag_pack": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "hb_diag_build_workspace_bytes": (c_size, [c_void_p, c_i64]),
    "hb_diag_build": (c_int, [c_void_p, c_void_p, c_i64, c_void_p, c_void_p, c_void_p, c_size, c_void_p]),
    "hb_normal_workspace_bytes": (c_size, [c_void_p, c_i64, c_i64]),
    "hb_toeplitz_apply": (c_int, [c_void_p, c_void_p, c_void_p, c_i64, c_i64, c_void_p, c_int, c_void_p,
                                  c_void_p, c_size, c_void_p]),
    "hb_sense_normal_apply": (c_int, [c_void_p, c_i64, c_void_p, c_void_p, c_void_p, P_i64, c_i64, c_void_p,
                                      P_i64, c_float, c_void_p, c_size, c_void_p]),
    "hb_systems_workspace_bytes": (c_size, [c_void_p, c_i64, c_i64, c_int]),
    "hb_sense_normal_apply_systems": (c_int, [c_void_p, c_i64, P_sys, c_void_p, c_size, c_void_p]),
    "hb_cg_run_systems": (c_int, [c_void_p, c_i64, P_sys, c_int, c_double, c_int, P_i32, P_i32, c_void_p, c_size,
                                  c_void_p]),
    "hb_cg_workspace_bytes": (c_size, [c_void_p, c_i64, c_i64, c_int]),
    "hb_cg_run": (c_int, [c_void_p, c_i64, c_void_p, c_void_p, c_void_p, P_i64, c_i64, c_void_p, P_i64,
                          c_float, c_int, c_double, P_i32, P_i32, c_void_p, c_size, c_void_p]),
    "hb_toeplitz_apply_noalloc": (c_int, [c_i64, c_i64, c_i64, c_void_p, c_void_p, c_i64, c_i64, c_void_p, c_int,
                                          c_void_p, c_void_p]),
    "hb_autotune_workspace_bytes": (c_size, [c_void_p, c_i64]),
    "hb_plan_plane_schedule": (ctypes.c_char_p, [c_void_p]),
    "hb_cg_batch_workspace_bytes": (c_size, [c_void_p, c_i64, c_i64]),
    "hb_cg_batch_create": (c_int, [ctypes.POINTER(c_void_p), c_void_p, c_i64, c_i64, c_void_p, c_size]),
    "hb_cg_batch_destroy": (c_int, [c_void_p]),
    "hb_cg_batch_add": (c_int, [c_void_p, c_void_p, c_int, c_double, ctypes.POINTER(c_i64)]),
    "hb_cg_batch_step": (c_int, [c_void_p, c_void_p, ctypes.POINTER(c_i64)]),
    "hb_cg_batch_retire": (c_int, [c_void_p, P_i64, P_i32, P_i32, c_i64, ctypes.POINTER(c_i64)]),
    "hb_plan_autotune": (c_int, [c_void_p, c_i64, c_void_p, c_size, c_void_p, ctypes.POINTER(c_int),
                                 ctypes.POINTER(c_double)]),
    "hb_nufft_create": (c_int, [ctypes.POINTER(c_void_p), c_i64, c_i64, c_i64, c_void_p, c_i64, c_double, c_int,
                                c_int, c_void_p]),
    "hb_nufft_destroy": (c_int, [c_void_p]),
    "hb_nufft_width": (c_int, [c_void_p]),
    "hb_nufft_type1": (c_int, [c_void_p, c_void_p, c_void_p, c_i64, c_int, c_void_p]),
    "hb_nufft_type2": (c_int, [c_void_p, c_void_p, c_void_p, c_i64, c_int, c_void_p]),
    "hb_sense_adjoint_nufft": (c_int, [c_void_p, c_void_p, c_void_p, P_i64, c_i64, c_void_p, c_void_p, c_int,
                                       c_void_p]),
    "hb_sense_normal_nufft": (c_int, [c_void_p, c_void_p, c_void_p, P_i64, c_i64, c_void_p, c_void_p, c_void_p,
                                      c_int, c_void_p]),
    "hb_diag_build_nufft": (c_int, [c_void_p, c_void_p, c_i64, c_double, c_void_p, c_void_p, c_void_p, c_void_p]),
    "hb_sense_forward_nufft": (c_int, [c_void_p, c_void_p, c_void_p, P_i64, c_i64, c_void_p, c_void_p]),
    "hb_precond_build": (c_int, [c_void_p, c_void_p, c_i64, c_double, c_void_p, P_i64, c_i64, c_float, c_void_p,
                                 c_void_p]),
    "hb_precond_apply": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "hb_svt_blocks": (c_int, [c_void_p, c_i64, c_i64, c_i64, c_i64, c_i64, c_i64, c_i64, c_i64, c_void_p, c_i64,
                              c_double, c_int, c_void_p]),
    "hb_admm_vectors": (c_int, [c_i64, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_float, c_void_p]),
    "hb_launch_count": (ctypes.c_uint64, []),
    "hb_profile_start": (c_int, []),
    "hb_profile_stop": (c_int, [ctypes.POINTER(c_double), P_i64, c_int]),
}

HB_KERNEL_KINDS = 6
KERNEL_NAMES = ["expand_fwd_x", "plane_yz", "inv_x_combine", "cg_update", "diag", "nufft"]

_lib = None


class HastyError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class NotPositiveDefinite(HastyError):
    pass


def load(path: str | None = None):
    """Load libhasty_b200.so (once) and attach the prototypes."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIBPATH
    if not os.path.exists(path):
        raise ImportError(
            f"hastycompute_b200: native library {path} is missing; build it with "
            f"`python -m hastycompute_b200.build` (there is no CPU fallback)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(code: int):
    if code != HB_OK:
        msg = load().hb_last_error().decode(errors="replace")
        if code == HB_ERR_NOT_PD:
            raise NotPositiveDefinite(code, msg)
        raise HastyError(code, msg)


def i64_array(values):
    values = list(int(v) for v in values)
    return (ctypes.c_int64 * max(1, len(values)))(*values)


def profile_start():
    check(load().hb_profile_start())


def profile_stop():
    """Returns {kernel kind name: (total ms, launches)} for the recorded region."""
    ms = (ctypes.c_double * HB_KERNEL_KINDS)()
    n = (ctypes.c_int64 * HB_KERNEL_KINDS)()
    check(load().hb_profile_stop(ms, n, HB_KERNEL_KINDS))
    return {KERNEL_NAMES[k]: (ms[k], n[k]) for k in range(HB_KERNEL_KINDS)}


def launch_count():
    return int(load().hb_launch_count())
