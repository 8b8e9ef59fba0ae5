"""Seeded synthetic scalar fields with the shapes and value distributions of the
benchmark workloads (no dataset is available offline, so these stand in for it).

* ``bumps_field``: sum of Gaussian bumps + low-wavenumber sin/cos products + small
  noise (the 384x384x256 float64 "Miranda-like" workload).
* ``grf_field``: Gaussian random field with a k^-5/3 power spectrum, optionally
  scaled to [-1, 1] or to unit variance, optionally with tanh shells (sharp fronts).
"""
from __future__ import annotations

import numpy as np


def bumps_field(nx: int, ny: int, nz: int, seed: int = 1234, n_bumps: int = 64,
                dtype=np.float64) -> np.ndarray:
    """Return a (nz, ny, nx) array (x fastest in memory)."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(nz, dtype=np.float64), np.arange(ny, dtype=np.float64),
                          np.arange(nx, dtype=np.float64), indexing="ij")
    f = np.zeros((nz, ny, nx), dtype=np.float64)
    cx = rng.uniform(0, nx, n_bumps)
    cy = rng.uniform(0, ny, n_bumps)
    cz = rng.uniform(0, nz, n_bumps)
    sig = rng.uniform(8, 40, n_bumps)
    amp = rng.normal(0.0, 1.0, n_bumps)
    for i in range(n_bumps):
        r2 = (x - cx[i]) ** 2 + (y - cy[i]) ** 2 + (z - cz[i]) ** 2
        f += amp[i] * np.exp(-r2 / (2.0 * sig[i] ** 2))
    for k in range(1, 5):
        f += 0.5 * np.sin(2 * np.pi * k * x / nx) * np.cos(2 * np.pi * k * y / ny) * \
            np.sin(2 * np.pi * k * z / max(nz, 1) + 0.3 * k) / k
    f += rng.normal(0.0, 1e-4, f.shape)
    return f.astype(dtype)


def grf_field(nx: int, ny: int, nz: int, seed: int = 7, scale: str = "range",
              n_fronts: int = 0, dtype=np.float32) -> np.ndarray:
    """k^-5/3 Gaussian random field, shape (nz, ny, nx).

    scale="range" maps to [-1, 1]; scale="unit" gives zero mean / unit variance.
    n_fronts adds tanh shells of width 2 cells (sharp fronts)."""
    rng = np.random.default_rng(seed)
    shape = (nz, ny, nx)
    noise = rng.standard_normal(shape).astype(np.float32)
    spec = np.fft.rfftn(noise)
    kz = np.fft.fftfreq(nz)[:, None, None]
    ky = np.fft.fftfreq(ny)[None, :, None]
    kx = np.fft.rfftfreq(nx)[None, None, :]
    k = np.sqrt(kx * kx + ky * ky + kz * kz)
    k[0, 0, 0] = 1.0
    # amplitude ~ k^(-5/3 / 2 - 1) in 3D so that the shell-integrated spectrum ~ k^-5/3
    amp = k ** (-(5.0 / 3.0 + 2.0) / 2.0)
    amp[0, 0, 0] = 0.0
    spec *= amp.astype(np.complex64 if spec.dtype == np.complex64 else spec.dtype)
    f = np.fft.irfftn(spec, s=shape).astype(np.float64)
    if n_fronts:
        zz = np.arange(nz, dtype=np.float64)[:, None, None]
        yy = np.arange(ny, dtype=np.float64)[None, :, None]
        xx = np.arange(nx, dtype=np.float64)[None, None, :]
        std = f.std() if f.std() > 0 else 1.0
        for _ in range(n_fronts):
            c = rng.uniform(0, 1, 3) * np.array([nx, ny, nz])
            r0 = rng.uniform(0.05, 0.3) * min(nx, ny, max(nz, 1))
            r = np.sqrt((xx - c[0]) ** 2 + (yy - c[1]) ** 2 + (zz - c[2]) ** 2)
            f += std * np.tanh((r - r0) / 2.0)
    if scale == "range":
        lo, hi = f.min(), f.max()
        f = 2.0 * (f - lo) / (hi - lo) - 1.0 if hi > lo else np.zeros_like(f)
    elif scale == "unit":
        s = f.std()
        f = (f - f.mean()) / (s if s > 0 else 1.0)
    return f.astype(dtype)


def grf_field_torch(nx: int, ny: int, nz: int, seed: int = 7, scale: str = "unit", n_fronts: int = 0,
                    device: str = "cuda", dtype=None):
    """GPU version of grf_field for large fields (e.g. 1024^3): a k^-5/3 Gaussian random
    field generated with torch.fft on the device, optional tanh shells (width 2 cells)."""
    import torch
    dtype = dtype or torch.float32
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    noise = torch.randn((nz, ny, nx), generator=g, device=device, dtype=torch.float32)
    spec = torch.fft.rfftn(noise)
    del noise
    kz = torch.fft.fftfreq(nz, device=device)[:, None, None]
    ky = torch.fft.fftfreq(ny, device=device)[None, :, None]
    kx = torch.fft.rfftfreq(nx, device=device)[None, None, :]
    k = torch.sqrt(kx * kx + ky * ky + kz * kz)
    k[0, 0, 0] = 1.0
    amp = k.pow(-(5.0 / 3.0 + 2.0) / 2.0)
    amp[0, 0, 0] = 0.0
    spec *= amp
    del k, amp
    f = torch.fft.irfftn(spec, s=(nz, ny, nx))
    del spec
    if n_fronts:
        cpu = torch.Generator()
        cpu.manual_seed(seed + 1)
        std = float(f.std())
        zz = torch.arange(nz, device=device, dtype=torch.float32)[:, None, None]
        yy = torch.arange(ny, device=device, dtype=torch.float32)[None, :, None]
        xx = torch.arange(nx, device=device, dtype=torch.float32)[None, None, :]
        for _ in range(n_fronts):
            c = torch.rand(3, generator=cpu) * torch.tensor([nx, ny, nz], dtype=torch.float32)
            r0 = float(0.05 + 0.25 * torch.rand(1, generator=cpu)) * min(nx, ny, max(nz, 1))
            r = torch.sqrt((xx - float(c[0])) ** 2 + (yy - float(c[1])) ** 2 + (zz - float(c[2])) ** 2)
            f += std * torch.tanh((r - r0) / 2.0)
            del r
    if scale == "range":
        lo, hi = f.min(), f.max()
        f = 2.0 * (f - lo) / (hi - lo) - 1.0
    elif scale == "unit":
        f = (f - f.mean()) / f.std()
    return f.to(dtype).contiguous()
