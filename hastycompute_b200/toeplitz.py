"""Python host layer over the C ABI, on torch device tensors.

Mirrors the reference operator semantics:

* ``ToeplitzPlan.build_diagonal`` / ``pack_diagonal`` -- ``CUDANormalNufftToeplitz``'s
  diagonal construction (``lib/fft/nufft.cpp:932-1053``) and the from-diagonal
  constructor (``nufft.cpp:1133-1161``).
* ``ToeplitzPlan.apply`` / ``apply_add`` / ``apply_addcmul`` / ``apply_inplace`` --
  ``nufft.cpp:1163-1197`` (``apply`` returns a view into ``storage2`` as the reference
  does).
* ``ToeplitzPlan.sense_normal`` -- ``sense_normal_apply`` with the Toeplitz body
  (``lib/mri/sense.ixx:500-578``), batched over systems and frames.
* ``ToeplitzPlan.cg`` -- ``ConjugateGradient::run`` (``lib/op/opalgs.cpp:50-96``) on
  ``A + lambda*I`` for many systems at once.

Every call goes to ``libhasty_b200.so``; there is no fallback.
"""
from __future__ import annotations

import ctypes

import torch

from . import capi


def _stream_ptr(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _check_c64(t, name, device, shape=None):
    if t.dtype != torch.complex64:
        raise RuntimeError(f"{name} must be complex64")
    if t.device != device:
        raise RuntimeError(f"{name} must reside on {device}")
    if not t.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")
    if shape is not None and tuple(t.shape[-len(shape):]) != tuple(shape):
        raise RuntimeError(f"{name} has shape {tuple(t.shape)}, expected (..., {shape})")


class System:
    """One system of a heterogeneous batch (``struct hb_system``).

    x: image [nz, ny, nx] (CG: initial guess, overwritten with the solution); out: the
    normal-op output; b: CG right-hand side; smaps: this system's coil maps; coils:
    indices into them (default all); packed: this system's packed diagonal (1-D view);
    lam: adds lam * x; precond: CG only, a circulant preconditioner from
    ``ToeplitzPlan.build_preconditioner`` (preconditioned CG for this system)."""

    def __init__(self, x, smaps, packed, out=None, b=None, coils=None, lam=0.0, precond=None):
        self.x, self.out, self.b, self.smaps, self.packed, self.lam = x, out, b, smaps, packed, float(lam)
        self.precond = precond
        self.coils = list(range(smaps.shape[0])) if coils is None else [int(c) for c in coils]


class ToeplitzPlan:
    """Geometry of an nz x ny x nx image and its 2x Toeplitz grid on one CUDA device."""

    def __init__(self, nmodes, device=None, precision="fp32"):
        self.lib = capi.load()
        if len(nmodes) == 4:  # reference convention [ntransf, nz, ny, nx]
            if nmodes[0] != 1:
                raise RuntimeError("only ntransf = 1 is supported")
            nmodes = nmodes[1:]
        self.shape = tuple(int(n) for n in nmodes)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        if self.device.type != "cuda":
            raise RuntimeError("ToeplitzPlan needs a CUDA device")
        idx = self.device.index if self.device.index is not None else torch.cuda.current_device()
        self.device = torch.device("cuda", idx)
        h = ctypes.c_void_p()
        capi.check(self.lib.hb_plan_create(ctypes.byref(h), *self.shape, idx))
        self._h = h
        self._ws = None
        if precision != "fp32":
            self.set_precision(precision)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self.lib.hb_plan_destroy(h)
            except Exception:
                pass
            self._h = None

    _PRECISIONS = {"fp32": capi.HB_PRECISION_FP32, "bf16x3": capi.HB_PRECISION_BF16X3}

    def set_precision(self, precision):
        """"fp32" (default): every pass on the CUDA cores in FP32.  "bf16x3": the forward x
        pass as a tensor-core contraction with BF16 hi + lo operands and FP32 accumulation
        (ny = nx = 128 only); the other passes stay FP32."""
        if precision not in self._PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(self._PRECISIONS)}, got {precision!r}")
        capi.check(self.lib.hb_plan_set_precision(self._h, self._PRECISIONS[precision]))

    @property
    def precision(self):
        code = int(self.lib.hb_plan_precision(self._h))
        return {v: k for k, v in self._PRECISIONS.items()}[code]

    def wait_status(self):
        """Raises if a tensor-core pass on this device gave up waiting (its output is then
        incomplete); clears the flag.  Synchronous."""
        capi.check(self.lib.hb_wait_status(self.device.index))

    @property
    def grid(self):
        return tuple(2 * n for n in self.shape)

    def packed_numel(self):
        return int(self.lib.hb_diag_packed_floats(self._h))

    def _workspace(self, nbytes):
        if self._ws is None or self._ws.numel() < nbytes:
            self._ws = torch.empty(int(nbytes), dtype=torch.uint8, device=self.device)
        return self._ws

    def cg_batch(self, max_systems, max_coil_slots):
        """A running batch of CG solves on this plan (continuous batching); see CgBatch."""
        return CgBatch(self, max_systems, max_coil_slots)

    def plane_schedule(self):
        """Name of the plane-pass schedule the next call launches (``hb_plan_plane_schedule``)."""
        return self.lib.hb_plan_plane_schedule(self._h).decode()

    def autotune(self, nslots=16):
        """Times the plane-pass schedules on nslots (system, coil) slots and keeps the
        fastest for this plan.  Returns (schedule index, ms per launch)."""
        nb = self.lib.hb_autotune_workspace_bytes(self._h, int(nslots))
        ws = torch.empty(int(nb), dtype=torch.uint8, device=self.device)
        chosen = ctypes.c_int(-1)
        ms = ctypes.c_double(0.0)
        capi.check(self.lib.hb_plan_autotune(self._h, int(nslots), _ptr(ws), nb, _stream_ptr(self.device),
                                             ctypes.byref(chosen), ctypes.byref(ms)))
        return chosen.value, ms.value

    # ---------------------------------------------------------------- diagonal ----
    def build_diagonal(self, coords, want_complex=False, method="exact", tol=1e-6, weights=None):
        """Construction of T from a trajectory coords [3, K] float32 (radians).

        method "exact": FP64 direct sum (``hb_diag_build``); "nufft": the reference's own
        construction through a type-1 NUFFT at tolerance ``tol`` (``hb_diag_build_nufft``,
        ``nufft.cpp:932-971``), much faster for long trajectories, optionally with sample
        ``weights`` (density compensation).
        Returns the packed diagonal (float32) and, if requested, the reference-layout
        complex64 T [2nz, 2ny, 2nx]."""
        if coords.dtype != torch.float32 or coords.dim() != 2 or coords.shape[0] != 3:
            raise RuntimeError("coords must be float32 [3, K]")
        coords = coords.to(self.device).contiguous()
        K = coords.shape[1]
        packed = torch.empty(self.packed_numel(), dtype=torch.float32, device=self.device)
        T = torch.empty(self.grid, dtype=torch.complex64, device=self.device) if want_complex else None
        if weights is not None:
            if method != "nufft":
                raise RuntimeError("sample weights need method='nufft'")
            weights = weights.to(self.device, torch.float32).reshape(-1).contiguous()
            if weights.numel() != K:
                raise RuntimeError("weights must hold one value per sample")
        if method == "nufft":
            capi.check(self.lib.hb_diag_build_nufft(self._h, _ptr(coords), K, float(tol), _ptr(weights), _ptr(packed),
                                                    _ptr(T), _stream_ptr(self.device)))
        elif method == "exact":
            nb = self.lib.hb_diag_build_workspace_bytes(self._h, K)
            ws = torch.empty(int(nb), dtype=torch.uint8, device=self.device)
            capi.check(self.lib.hb_diag_build(self._h, _ptr(coords), K, _ptr(packed), _ptr(T), _ptr(ws), nb,
                                              _stream_ptr(self.device)))
        else:
            raise RuntimeError(f"unknown diagonal method {method!r} (exact or nufft)")
        return (packed, T) if want_complex else packed

    def pack_diagonal(self, T):
        """Pack a reference-layout diagonal [(1,) 2nz, 2ny, 2nx] complex64."""
        T = T.reshape(self.grid)
        _check_c64(T, "diagonal", self.device, self.grid)
        packed = torch.empty(self.packed_numel(), dtype=torch.float32, device=self.device)
        capi.check(self.lib.hb_diag_pack(self._h, _ptr(T), _ptr(packed), _stream_ptr(self.device)))
        return packed

    # ------------------------------------------------------- Toeplitz normal op ----
    def _toeplitz(self, x, out, ldz, ldy, mul, accumulate, packed):
        _check_c64(x, "in", self.device, self.shape)
        if mul is not None:
            _check_c64(mul, "mul", self.device, self.shape)
        nb = self.lib.hb_normal_workspace_bytes(self._h, 1, 1)
        ws = self._workspace(nb)
        capi.check(self.lib.hb_toeplitz_apply(self._h, _ptr(x), _ptr(out), ldz, ldy, _ptr(mul), int(accumulate),
                                              _ptr(packed), _ptr(ws), nb, _stream_ptr(self.device)))

    def apply(self, x, packed, storage2=None):
        """``apply`` (nufft.cpp:1163-1170): the result is written into storage2 (2x grid)
        and the cropped view [:nz, :ny, :nx] of it is returned."""
        if storage2 is None:
            storage2 = torch.empty((1,) + self.grid, dtype=torch.complex64, device=self.device)
        s2 = storage2.reshape(self.grid)
        _check_c64(s2, "storage2", self.device, self.grid)
        M0, M1, M2 = self.grid
        self._toeplitz(x, s2, M1 * M2, M2, None, 0, packed)
        view = storage2[..., : self.shape[0], : self.shape[1], : self.shape[2]]
        return view

    def apply_add(self, x, add_to, packed):
        _check_c64(add_to, "add_to", self.device, self.shape)
        n0, n1, n2 = self.shape
        self._toeplitz(x, add_to, n1 * n2, n2, None, 1, packed)

    def apply_addcmul(self, x, add_to, mul, packed):
        _check_c64(add_to, "add_to", self.device, self.shape)
        n0, n1, n2 = self.shape
        self._toeplitz(x, add_to, n1 * n2, n2, mul, 1, packed)

    def apply_inplace(self, x, packed):
        n0, n1, n2 = self.shape
        self._toeplitz(x, x, n1 * n2, n2, None, 0, packed)

    # ------------------------------------------------------------ SENSE normal ----
    def sense_normal(self, x, out, smaps, packed, coils=None, diag_index=None, lam=0.0, workspace_bytes=None):
        """out[s] = sum_c conj(S_c) Top_{d(s)}(S_c x[s]) + lam x[s] for every system s.

        x, out: [nsys, nz, ny, nx] (or [nz, ny, nx]); smaps [C, nz, ny, nx];
        packed: one packed diagonal or [ndiag, packed]; diag_index: per system."""
        x4 = x.reshape((-1,) + self.shape)
        out4 = out.reshape((-1,) + self.shape)
        _check_c64(x4, "in", self.device, self.shape)
        _check_c64(out4, "out", self.device, self.shape)
        _check_c64(smaps, "smaps", self.device, self.shape)
        nsys = x4.shape[0]
        if coils is None:
            coils = list(range(smaps.shape[0]))
        if any(c < 0 or c >= smaps.shape[0] for c in coils):
            raise RuntimeError("coil index out of range")
        self._check_packed(packed, diag_index, nsys)
        ca = capi.i64_array(coils)
        da = capi.i64_array(diag_index) if diag_index is not None else None
        nb = self.lib.hb_normal_workspace_bytes(self._h, nsys, len(coils))
        if workspace_bytes is not None:
            nb = min(nb, int(workspace_bytes))
        ws = self._workspace(nb)
        capi.check(self.lib.hb_sense_normal_apply(self._h, nsys, _ptr(x4), _ptr(out4), _ptr(smaps), ca, len(coils),
                                                  _ptr(packed), da, float(lam), _ptr(ws), nb,
                                                  _stream_ptr(self.device)))
        return out

    def _check_packed(self, packed, diag_index, nsys):
        if packed.dtype != torch.float32 or not packed.is_contiguous() or packed.device != self.device:
            raise RuntimeError("packed diagonal must be a contiguous float32 tensor on the plan's device")
        nd = packed.numel() // self.packed_numel()
        if nd * self.packed_numel() != packed.numel() or nd < 1:
            raise RuntimeError("packed diagonal has the wrong size")
        if diag_index is not None:
            if len(diag_index) != nsys:
                raise RuntimeError("diag_index must have one entry per system")
            if any(d < 0 or d >= nd for d in diag_index):
                raise RuntimeError("diag_index out of range")

    # ---------------------------------------------------------------------- CG ----
    def cg(self, x, b, smaps, packed, iters=30, tol=0.0, lam=0.0, coils=None, diag_index=None,
           workspace_bytes=None, raise_not_pd=True):
        """Batched CG (opalgs.cpp:50-96) on (A^H A)_toep + lam I; x is updated in place.

        Returns (status, iters_done) as lists (one per system)."""
        x4 = x.reshape((-1,) + self.shape)
        b4 = b.reshape((-1,) + self.shape)
        _check_c64(x4, "x", self.device, self.shape)
        _check_c64(b4, "b", self.device, self.shape)
        _check_c64(smaps, "smaps", self.device, self.shape)
        nsys = x4.shape[0]
        if b4.shape[0] != nsys:
            raise RuntimeError("x and b must hold the same number of systems")
        if coils is None:
            coils = list(range(smaps.shape[0]))
        self._check_packed(packed, diag_index, nsys)
        ca = capi.i64_array(coils)
        da = capi.i64_array(diag_index) if diag_index is not None else None
        nb = self.lib.hb_cg_workspace_bytes(self._h, nsys, len(coils), int(iters))
        if workspace_bytes is not None:
            nb = min(nb, int(workspace_bytes))
        ws = self._workspace(max(nb, 1))
        status = (ctypes.c_int32 * nsys)()
        done = (ctypes.c_int32 * nsys)()
        code = self.lib.hb_cg_run(self._h, nsys, _ptr(x4), _ptr(b4), _ptr(smaps), ca, len(coils), _ptr(packed), da,
                                  float(lam), int(iters), float(tol), status, done, _ptr(ws), nb,
                                  _stream_ptr(self.device))
        if code == capi.HB_ERR_NOT_PD and not raise_not_pd:
            return list(status), list(done)
        capi.check(code)
        return list(status), list(done)

    # ------------------------------------------------------ circulant preconditioner ----
    def numel(self):
        n0, n1, n2 = self.shape
        return n0 * n1 * n2

    def build_preconditioner(self, coords, smaps, coils=None, lam=0.0, tol=1e-6):
        """Circulant preconditioner (``CirculantPreconditionerOp::build_diagonal``,
        ``lib/mri/precond.cpp:65-117``; ``torch_precond.py:60-105``) of sum_c S_c^H A^H A S_c
        + lam I for a trajectory coords [3, K] float32: float32 [nz, ny, nx] in FFT order."""
        if coords.dtype != torch.float32 or coords.dim() != 2 or coords.shape[0] != 3:
            raise RuntimeError("coords must be float32 [3, K]")
        coords = coords.to(self.device).contiguous()
        _check_c64(smaps, "smaps", self.device, self.shape)
        coils = list(range(smaps.shape[0])) if coils is None else [int(c) for c in coils]
        if not coils or any(c < 0 or c >= smaps.shape[0] for c in coils):
            raise RuntimeError("coil index out of range")
        out = torch.empty(self.shape, dtype=torch.float32, device=self.device)
        capi.check(self.lib.hb_precond_build(self._h, _ptr(coords), coords.shape[1], float(tol), _ptr(smaps),
                                             capi.i64_array(coils), len(coils), float(lam), _ptr(out),
                                             _stream_ptr(self.device)))
        return out

    def apply_preconditioner(self, precond, x, out=None):
        """out = P x = IFFT(precond * FFT(x)) (``CirculantPreconditionerOp::apply``, precond.cpp:30-52)."""
        _check_c64(x, "x", self.device, self.shape)
        if out is None:
            out = torch.empty_like(x)
        _check_c64(out, "out", self.device, self.shape)
        if precond.dtype != torch.float32 or precond.numel() != self.numel() or not precond.is_contiguous():
            raise RuntimeError("precond must be a contiguous float32 [nz, ny, nx] tensor")
        capi.check(self.lib.hb_precond_apply(self._h, _ptr(precond), _ptr(x), _ptr(out), _stream_ptr(self.device)))
        return out

    def cg_host(self, x_host, b_host, smaps, packed, iters=30, tol=0.0, lam=0.0, coils=None, diag_index=None,
                chunks=4, raise_not_pd=True, out_host=None):
        """CG for systems whose initial guess and right-hand side live in (pinned) host memory;
        the solution is written into ``out_host`` (default: back into ``x_host``).  The systems are solved in ``chunks``
        consecutive groups: all host-to-device copies are issued first on a copy stream, each
        group's solve waits only for its own data, and each group's solution is copied back
        while the next group is solved, so the copy engines work beside the SMs (the
        reference copies every inner batch to and from the host synchronously,
        ``batch_sense.cpp:349-450``).  Returns (status, iters_done) as lists."""
        x4 = x_host.reshape((-1,) + self.shape)
        b4 = b_host.reshape((-1,) + self.shape)
        o4 = x4 if out_host is None else out_host.reshape((-1,) + self.shape)
        nsys = x4.shape[0]
        if o4.shape[0] != nsys:
            raise RuntimeError("out_host must hold every system")
        if b4.shape[0] != nsys or x4.dtype != torch.complex64 or b4.dtype != torch.complex64:
            raise RuntimeError("x_host and b_host must be complex64 with the same number of systems")
        if diag_index is None:
            diag_index = [0] * nsys
        main = torch.cuda.current_stream(self.device)
        if getattr(self, "_copy_stream", None) is None:
            self._copy_stream = torch.cuda.Stream(self.device)
        cs = self._copy_stream
        xd = torch.empty(x4.shape, dtype=torch.complex64, device=self.device)
        bd = torch.empty(b4.shape, dtype=torch.complex64, device=self.device)
        bounds = [round(k * nsys / max(1, chunks)) for k in range(max(1, chunks) + 1)]
        ready = []
        cs.wait_stream(main)  # the device buffers may be reused memory
        with torch.cuda.stream(cs):
            for k in range(len(bounds) - 1):
                sl = slice(bounds[k], bounds[k + 1])
                xd[sl].copy_(x4[sl], non_blocking=True)
                bd[sl].copy_(b4[sl], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(cs)
                ready.append(ev)
        status, done = [], []
        try:
            for k in range(len(bounds) - 1):
                lo, hi = bounds[k], bounds[k + 1]
                if hi <= lo:
                    continue
                main.wait_event(ready[k])
                st, it = self.cg(xd[lo:hi], bd[lo:hi], smaps, packed, iters=iters, tol=tol, lam=lam, coils=coils,
                                 diag_index=list(diag_index[lo:hi]), raise_not_pd=raise_not_pd)
                status += st
                done += it
                cs.wait_stream(main)
                with torch.cuda.stream(cs):
                    o4[lo:hi].copy_(xd[lo:hi], non_blocking=True)
        finally:
            main.wait_stream(cs)
            xd.record_stream(cs)
            bd.record_stream(cs)
        return status, done

    # ------------------------------------------------------- heterogeneous batch ----
    def _systems(self, systems, cg):
        arr = (capi.HbSystem * len(systems))()
        keep = []
        for i, q in enumerate(systems):
            _check_c64(q.x, "x", self.device, self.shape)
            _check_c64(q.smaps, "smaps", self.device, self.shape)
            if cg:
                _check_c64(q.b, "b", self.device, self.shape)
            else:
                _check_c64(q.out, "out", self.device, self.shape)
            if q.packed.dtype != torch.float32 or q.packed.numel() != self.packed_numel() or \
                    not q.packed.is_contiguous() or q.packed.device != self.device:
                raise RuntimeError("each system needs one contiguous float32 packed diagonal on the device")
            if any(c < 0 or c >= q.smaps.shape[0] for c in q.coils) or not q.coils:
                raise RuntimeError("coil index out of range")
            ca = capi.i64_array(q.coils)
            keep.append(ca)
            arr[i].x = q.x.data_ptr()
            arr[i].out = q.out.data_ptr() if q.out is not None else None
            arr[i].b = q.b.data_ptr() if q.b is not None else None
            arr[i].smaps = q.smaps.data_ptr()
            arr[i].coils = ca
            arr[i].ncoil = len(q.coils)
            arr[i].packed_diag = q.packed.data_ptr()
            arr[i].lam = q.lam
            pc = getattr(q, "precond", None)
            if pc is not None:
                if not cg:
                    raise RuntimeError("a preconditioner only applies to CG systems")
                if pc.dtype != torch.float32 or pc.numel() != self.numel() or not pc.is_contiguous() or \
                        pc.device != self.device:
                    raise RuntimeError("precond must be a contiguous float32 [nz, ny, nx] tensor on the device")
                arr[i].precond = pc.data_ptr()
        return arr, keep

    def sense_normal_systems(self, systems, workspace_bytes=None):
        """out = (A^H A)_toep x + lam x for every System, in as few launch sequences as the workspace allows."""
        arr, keep = self._systems(systems, cg=False)
        ncoil = sum(len(q.coils) for q in systems)
        nb = self.lib.hb_systems_workspace_bytes(self._h, len(systems), ncoil, -1)
        if workspace_bytes is not None:
            nb = min(nb, int(workspace_bytes))
        ws = self._workspace(nb)
        capi.check(self.lib.hb_sense_normal_apply_systems(self._h, len(systems), arr, _ptr(ws), nb,
                                                          _stream_ptr(self.device)))

    def cg_systems(self, systems, iters=30, tol=0.0, graph=True, workspace_bytes=None, raise_not_pd=True):
        """Batched CG over heterogeneous systems; each System's x is updated in place.
        graph=True captures each iteration as a CUDA graph and replays it."""
        arr, keep = self._systems(systems, cg=True)
        n = len(systems)
        ncoil = sum(len(q.coils) for q in systems)
        nb = self.lib.hb_systems_workspace_bytes(self._h, n, ncoil, int(iters))
        if workspace_bytes is not None:
            nb = min(nb, int(workspace_bytes))
        ws = self._workspace(max(nb, 1))
        status = (ctypes.c_int32 * n)()
        done = (ctypes.c_int32 * n)()
        code = self.lib.hb_cg_run_systems(self._h, n, arr, int(iters), float(tol),
                                          capi.HB_CG_GRAPH if graph else 0, status, done, _ptr(ws), nb,
                                          _stream_ptr(self.device))
        if code == capi.HB_ERR_NOT_PD and not raise_not_pd:
            return list(status), list(done)
        capi.check(code)
        return list(status), list(done)


class CgBatch:
    """A running batch of CG solves on one plan (``hb_cg_batch_*``): systems join at the
    next iteration boundary (``add``), every ``step`` runs one launch sequence in which the
    new systems initialise and every other member takes one CG iteration, and systems
    leave when they converge, break down or have run their own iteration budget
    (``retire``).  A member's iterates are bitwise those of ``ToeplitzPlan.cg_systems`` on
    the same system, whatever else is in the batch.

    Replaces the reference's thread-pool fan-out of independent CG solves
    (``BatchedConjugateGradient::run``, ``lib/op/opalgs.ixx:93-121``) with continuous
    batching on the device."""

    def __init__(self, plan, max_systems, max_coil_slots):
        self.plan = plan
        self.lib = plan.lib
        nb = int(self.lib.hb_cg_batch_workspace_bytes(plan._h, int(max_systems), int(max_coil_slots)))
        self._ws = torch.empty(nb, dtype=torch.uint8, device=plan.device)
        h = ctypes.c_void_p()
        capi.check(self.lib.hb_cg_batch_create(ctypes.byref(h), plan._h, int(max_systems), int(max_coil_slots),
                                               _ptr(self._ws), nb))
        self._h = h
        self._keep = {}  # handle -> tensors and coil arrays the device reads until retirement
        self.max_systems = int(max_systems)
        self.max_coil_slots = int(max_coil_slots)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self.lib.hb_cg_batch_destroy(h)
            except Exception:
                pass
            self._h = None

    def add(self, system, iters, tol=0.0):
        """Queues a System (x: initial guess in, solution out; b; coils; packed; lam).
        Returns its handle; raises HastyError (HB_ERR_WORKSPACE) when the batch is full."""
        arr, keep = self.plan._systems([system], cg=True)
        hd = ctypes.c_int64(-1)
        capi.check(self.lib.hb_cg_batch_add(self._h, arr, int(iters), float(tol), ctypes.byref(hd)))
        self._keep[hd.value] = (system, keep)
        return hd.value

    def step(self, stream=None):
        """One iteration boundary; returns the number of systems still in the batch."""
        n = ctypes.c_int64(0)
        sp = ctypes.c_void_p(stream.cuda_stream) if stream is not None else _stream_ptr(self.plan.device)
        capi.check(self.lib.hb_cg_batch_step(self._h, sp, ctypes.byref(n)))
        return int(n.value)

    def retire(self):
        """Systems that left the batch since the last call: [(handle, status, iterations)]."""
        cap = self.max_systems * 4 + 16
        hs = (ctypes.c_int64 * cap)()
        st = (ctypes.c_int32 * cap)()
        it = (ctypes.c_int32 * cap)()
        n = ctypes.c_int64(0)
        capi.check(self.lib.hb_cg_batch_retire(self._h, hs, st, it, cap, ctypes.byref(n)))
        out = [(int(hs[i]), int(st[i]), int(it[i])) for i in range(n.value)]
        for hd, _, _ in out:
            self._keep.pop(hd, None)
        return out
