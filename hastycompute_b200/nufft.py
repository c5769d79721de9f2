"""Non-uniform FFT (types 1 and 2) and the SENSE forward/adjoint operators, over the C ABI.

Mirrors the reference's NUFFT front end:

* ``NufftType`` / ``NufftOptions`` -- ``lib/fft/nufft.ixx:20-70`` (type 1 defaults to the
  positive sign, type 2 to the negative one, tolerance 1e-5);
* ``CUDANufft(coords, nmodes, opts).apply(in, out)`` -- ``nufft.ixx:108-160`` /
  ``nufft.cpp:540-767`` with ``nmodes = [ntransf, nz, ny, nx]``: type 1 maps
  ``in [ntransf, nfreq]`` to ``out [ntransf, nz, ny, nx]``, type 2 the reverse;
* ``NufftPlan.sense_adjoint`` / ``sense_forward`` / ``sense_normal`` -- the coil loops of the
  SENSE operators built on those plans (``lib/mri/sense.ixx:426-497``), the normal one with
  the k-space manipulators of ``batch_sense.cpp:452-486``; ``sense_adjoint`` gives the CG
  right-hand side ``b = sum_c conj(S_c) NUFFT^H(y_c)``.

Only 3-D transforms are compiled (the path's images are 3-D); ``2 * N`` per axis must be
one of 8, 16, 32, 64, 128, 256, 512, 96, 160, 192, 320.  Every call runs the sm_100a kernels of
``libhasty_b200.so``; there is no fallback.
"""
from __future__ import annotations

import ctypes
import enum

import torch

from . import capi
from .toeplitz import _check_c64, _ptr, _stream_ptr


class NufftType(enum.IntEnum):
    eType1 = 1  # adjoint: nonuniform -> modes
    eType2 = 2  # forward: modes -> nonuniform


class NufftOptions:
    """``hasty::fft::NufftOptions`` (``nufft.ixx:26-70``)."""

    def __init__(self, type=NufftType.eType1, positive=True, tol=1e-5):
        self.type = NufftType(type)
        self.positive = bool(positive)
        self.tol = float(tol)

    @classmethod
    def type1(cls, positive=True, tol=1e-5):
        return cls(NufftType.eType1, positive, tol)

    @classmethod
    def type2(cls, positive=False, tol=1e-5):
        return cls(NufftType.eType2, positive, tol)

    def get_positive(self):
        return 1 if self.positive else -1


class NufftPlan:
    """A plan for modes ``nmodes`` = (nz, ny, nx), (ny, nx) or (nx,) at fixed sample
    coordinates (``hb_nufft``): coords float32 [len(nmodes), nsamples] on a CUDA device, row
    a pairing with image axis a (the reference's 1-D, 2-D and 3-D plans)."""

    def __init__(self, coords, nmodes, tol=1e-5, maxbatch=8):
        self.lib = capi.load()
        self.shape = tuple(int(n) for n in nmodes)
        d = len(self.shape)
        if d not in (1, 2, 3) or coords.dim() != 2 or coords.shape[0] != d:
            raise RuntimeError("coords must be [ndim, nsamples] with ndim = len(nmodes) in 1..3")
        if coords.dtype != torch.float32 or coords.device.type != "cuda":
            raise RuntimeError("coords must be float32 on a CUDA device")
        if d < 3 and 1 in self.shape:
            raise RuntimeError("a transformed axis needs more than one mode")
        self.coords = coords.contiguous()
        self.device = self.coords.device
        self.nfreq = int(coords.shape[1])
        self._h = None
        h = ctypes.c_void_p()
        dims3 = (1,) * (3 - d) + self.shape  # leading axes of length 1 select the 2-D / 1-D plan
        capi.check(self.lib.hb_nufft_create(ctypes.byref(h), *dims3, _ptr(self.coords), self.nfreq,
                                            float(tol), int(maxbatch), self.device.index, _stream_ptr(self.device)))
        self._h = h

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self.lib.hb_nufft_destroy(h)
        self._h = None

    __del__ = close

    @property
    def width(self):
        return int(self.lib.hb_nufft_width(self._h))

    def type1(self, c, f=None, isign=+1):
        """f[t] = sum_j c[t, j] exp(isign i k.x_j); c [ntransf, nfreq] -> f [ntransf, nz, ny, nx]."""
        c = c.reshape(-1, self.nfreq)
        _check_c64(c, "c", self.device)
        if f is None:
            f = torch.empty((c.shape[0],) + self.shape, dtype=torch.complex64, device=self.device)
        _check_c64(f, "f", self.device, self.shape)
        capi.check(self.lib.hb_nufft_type1(self._h, _ptr(c), _ptr(f), c.shape[0], int(isign),
                                           _stream_ptr(self.device)))
        return f

    def type2(self, f, c=None, isign=-1):
        """c[t, j] = sum_k f[t, k] exp(isign i k.x_j); f [ntransf, nz, ny, nx] -> c [ntransf, nfreq]."""
        f = f.reshape((-1,) + self.shape)
        _check_c64(f, "f", self.device, self.shape)
        if c is None:
            c = torch.empty((f.shape[0], self.nfreq), dtype=torch.complex64, device=self.device)
        _check_c64(c, "c", self.device, (self.nfreq,))
        capi.check(self.lib.hb_nufft_type2(self._h, _ptr(f), _ptr(c), f.shape[0], int(isign),
                                           _stream_ptr(self.device)))
        return c

    def sense_adjoint(self, kdata, smaps, coils=None, out=None, accumulate=False, weights=None):
        """out (+)= sum_b conj(smaps[coils[b]]) * type1(w * kdata[b]) (w: optional float32
        [nfreq] sample weights)."""
        coils = list(range(smaps.shape[0])) if coils is None else [int(c) for c in coils]
        kdata = kdata.reshape(len(coils), self.nfreq)
        _check_c64(kdata, "kdata", self.device)
        _check_c64(smaps, "smaps", self.device, self.shape)
        if out is None:
            out = torch.empty(self.shape, dtype=torch.complex64, device=self.device)
            accumulate = False
        _check_c64(out, "out", self.device, self.shape)
        if weights is not None:
            weights = weights.reshape(-1)
            if weights.dtype != torch.float32 or weights.numel() != self.nfreq or weights.device != self.device \
                    or not weights.is_contiguous():
                raise RuntimeError("weights must be a contiguous float32 [nfreq] tensor on the device")
        arr = (ctypes.c_int64 * max(1, len(coils)))(*coils)
        capi.check(self.lib.hb_sense_adjoint_nufft(self._h, _ptr(kdata), _ptr(smaps), arr, len(coils), _ptr(weights),
                                                   _ptr(out), 1 if accumulate else 0, _stream_ptr(self.device)))
        return out

    def sense_normal(self, x, smaps, coils=None, kdata=None, weights=None, out=None, accumulate=False):
        """out (+)= sum_b conj(S[c_b]) type1(w * (type2(S[c_b] x) - kdata[c_b])) -- the normal
        operator with the reference's k-space manipulators (``batch_sense.cpp:452-486``);
        kdata [C, nfreq] indexed by coil number, weights [nfreq] float32, both optional."""
        coils = list(range(smaps.shape[0])) if coils is None else [int(c) for c in coils]
        _check_c64(x, "x", self.device, self.shape)
        _check_c64(smaps, "smaps", self.device, self.shape)
        if kdata is not None:
            kdata = kdata.reshape(-1, self.nfreq)
            _check_c64(kdata, "kdata", self.device)
            if kdata.shape[0] <= max(coils):
                raise RuntimeError("kdata must hold a row for every coil index")
        if weights is not None:
            weights = weights.reshape(-1)
            if weights.dtype != torch.float32 or weights.numel() != self.nfreq or weights.device != self.device \
                    or not weights.is_contiguous():
                raise RuntimeError("weights must be a contiguous float32 [nfreq] tensor on the device")
        if out is None:
            out = torch.empty(self.shape, dtype=torch.complex64, device=self.device)
            accumulate = False
        _check_c64(out, "out", self.device, self.shape)
        arr = (ctypes.c_int64 * max(1, len(coils)))(*coils)
        capi.check(self.lib.hb_sense_normal_nufft(self._h, _ptr(x), _ptr(smaps), arr, len(coils), _ptr(kdata),
                                                  _ptr(weights), _ptr(out), 1 if accumulate else 0,
                                                  _stream_ptr(self.device)))
        return out

    def sense_forward(self, x, smaps, coils=None, kdata=None):
        """kdata[b] = type2(smaps[coils[b]] * x)."""
        coils = list(range(smaps.shape[0])) if coils is None else [int(c) for c in coils]
        _check_c64(x, "x", self.device, self.shape)
        _check_c64(smaps, "smaps", self.device, self.shape)
        if kdata is None:
            kdata = torch.empty((len(coils), self.nfreq), dtype=torch.complex64, device=self.device)
        _check_c64(kdata, "kdata", self.device, (self.nfreq,))
        arr = (ctypes.c_int64 * max(1, len(coils)))(*coils)
        capi.check(self.lib.hb_sense_forward_nufft(self._h, _ptr(x), _ptr(smaps), arr, len(coils), _ptr(kdata),
                                                   _stream_ptr(self.device)))
        return kdata


class CUDANufft:
    """``hasty::fft::CUDANufft`` (``nufft.ixx:108-160``): ``nmodes = [ntransf, nz, ny, nx]``,
    ``[ntransf, ny, nx]`` or ``[ntransf, nx]`` with coords [3|2|1, nfreq]."""

    def __init__(self, coords, nmodes, opts=None):
        opts = NufftOptions() if opts is None else opts
        if len(nmodes) not in (2, 3, 4):
            raise RuntimeError("nmodes must be [ntransf, nz, ny, nx], [ntransf, ny, nx] or [ntransf, nx]")
        self._ntransf = int(nmodes[0])
        self._nmodes = [int(n) for n in nmodes]
        self._opts = opts
        self._plan = NufftPlan(coords, nmodes[1:], tol=opts.tol, maxbatch=max(1, min(self._ntransf, 16)))

    def apply(self, inp, out):
        if self._opts.type == NufftType.eType1:
            if list(out.shape) != self._nmodes:
                raise RuntimeError("out.sizes() must equal nmodes given at construct")
            if tuple(inp.shape) != (self._ntransf, self._plan.nfreq):
                raise RuntimeError("in tensor must match ntransf in first dim and nfreq in second dim")
            self._plan.type1(inp, out, self._opts.get_positive())
        else:
            if list(inp.shape) != self._nmodes:
                raise RuntimeError("in.sizes() must equal nmodes given at construct")
            if tuple(out.shape) != (self._ntransf, self._plan.nfreq):
                raise RuntimeError("out tensor must match ntransf in first dim and nfreq in second dim")
            self._plan.type2(inp, out, self._opts.get_positive())

    def nfreq(self):
        return self._plan.nfreq

    def ndim(self):
        return len(self._nmodes) - 1

    def close(self):
        self._plan.close()
