"""Seeded synthetic inputs with the shapes and distributions of the benchmark workloads.

The reference reconstructs private HDF5 scans; these generators stand in for them:

* ``kooshball``: 3D radial trajectory, golden-means (2D golden-angle) spoke ordering,
  samples spanning [-pi, pi) along each spoke; ``frame``/``nframes`` interleave spokes
  across cardiac frames.  Returned as float32 [3, spokes*samples], row a <-> image axis a.
* ``coil_maps``: smooth complex Gaussian-blob sensitivities centred on a ring in the
  axial plane at 0.35 FOV, sigma ~ 0.3 FOV, smooth random phase, normalised so that
  sum_c |S_c|^2 = 1 per voxel.
* ``gaussian_image``: i.i.d. complex Gaussian image.
* ``flow_phantom``: smooth ellipsoid magnitude x exp(i * random linear phase per
  velocity encoding) + complex Gaussian noise.
"""
from __future__ import annotations

import numpy as np

GOLDEN_1 = 0.4656274277  # 2D golden means (Chan et al., 3D radial ordering)
GOLDEN_2 = 0.6823278038


def kooshball(nspokes, nsamples, frame=0, nframes=1, dtype=np.float32):
    i = np.arange(nspokes, dtype=np.float64) * nframes + frame
    cz = np.mod(i * GOLDEN_1, 1.0) * 2.0 - 1.0
    phi = 2.0 * np.pi * np.mod(i * GOLDEN_2, 1.0)
    sz = np.sqrt(np.maximum(0.0, 1.0 - cz * cz))
    d = np.stack([cz, sz * np.sin(phi), sz * np.cos(phi)], axis=0)  # [3, spokes] (z, y, x)
    t = -np.pi + 2.0 * np.pi * np.arange(nsamples, dtype=np.float64) / nsamples
    c = d[:, :, None] * t[None, None, :]
    return np.ascontiguousarray(c.reshape(3, -1).astype(dtype))


def _grid(shape):
    axes = [np.linspace(-0.5, 0.5, n, endpoint=False) + 0.5 / n for n in shape]
    return np.meshgrid(*axes, indexing="ij")


def coil_maps(ncoil, shape, seed=0, dtype=np.complex64):
    rng = np.random.default_rng(seed)
    z, y, x = _grid(shape)
    maps = np.empty((ncoil,) + tuple(shape), np.complex128)
    sigma = 0.3
    for c in range(ncoil):
        ang = 2.0 * np.pi * c / ncoil
        cy, cx = 0.35 * np.sin(ang), 0.35 * np.cos(ang)
        cz = 0.1 * rng.standard_normal()
        mag = np.exp(-((z - cz) ** 2 + (y - cy) ** 2 + (x - cx) ** 2) / (2 * sigma * sigma))
        g = rng.standard_normal(4)
        phase = g[0] * np.pi + 1.5 * (g[1] * z + g[2] * y + g[3] * x)
        maps[c] = mag * np.exp(1j * phase)
    norm = np.sqrt(np.sum(np.abs(maps) ** 2, axis=0))
    maps /= norm[None]
    return maps.astype(dtype)


def gaussian_image(shape, seed=0, dtype=np.complex64):
    rng = np.random.default_rng(seed)
    return ((rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2.0)).astype(dtype)


def flow_phantom(shape, nenc, seed=0, noise=1e-3, dtype=np.complex64):
    rng = np.random.default_rng(seed)
    z, y, x = _grid(shape)
    mag = np.exp(-np.maximum(0.0, (z / 0.35) ** 2 + (y / 0.4) ** 2 + (x / 0.3) ** 2 - 1.0) * 8.0)
    out = np.empty((nenc,) + tuple(shape), np.complex128)
    for e in range(nenc):
        g = rng.standard_normal(3)
        out[e] = mag * np.exp(1j * np.pi * (g[0] * z + g[1] * y + g[2] * x))
        out[e] += noise * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2.0)
    return out.astype(dtype)


def coil_maps_torch(ncoil, shape, seed=0, device="cuda"):
    """coil_maps() generated on the device (same construction), for large job pools."""
    import torch

    g = np.random.default_rng(seed)
    axes = [torch.linspace(-0.5, 0.5, n + 1, dtype=torch.float64, device=device)[:-1] + 0.5 / n for n in shape]
    z, y, x = torch.meshgrid(*axes, indexing="ij")
    maps = torch.empty((ncoil,) + tuple(shape), dtype=torch.complex128, device=device)
    sigma = 0.3
    for c in range(ncoil):
        ang = 2.0 * np.pi * c / ncoil
        cy, cx = 0.35 * np.sin(ang), 0.35 * np.cos(ang)
        cz = 0.1 * g.standard_normal()
        mag = torch.exp(-((z - cz) ** 2 + (y - cy) ** 2 + (x - cx) ** 2) / (2 * sigma * sigma))
        r = g.standard_normal(4)
        phase = r[0] * np.pi + 1.5 * (r[1] * z + r[2] * y + r[3] * x)
        maps[c] = mag * torch.exp(1j * phase)
    norm = torch.sqrt((maps.abs() ** 2).sum(0))
    return (maps / norm).to(torch.complex64).contiguous()
