"""Differentiable decode: the real-valued decode operator D (dequantised coefficients -> grid)
and its adjoint, over the C ABI (idx2g_coeffs / idx2g_synth / idx2g_synth_adjoint), wrapped in
a torch.autograd.Function so that gradients of a loss on the decoded grid flow to the
coefficients.

D is the reference decode (Core/idx2Decode.cpp:141-320) with the integer inverse zfp replaced
by its real form (Core/Zfp.h:181 ILift, exact halvings); it is linear, so the backward pass is
the adjoint kernel applied to the incoming gradient: nothing from the forward pass is stored,
each level is recomputed from the level gradients.

Coefficient tensor layout (per field): levels 0 (finest) to L-1, bricks row-major (x fastest)
on each level, 33^3 values per brick (33^2 for 2D) indexed (z*33 + y)*33 + x; see
include/idx2g.h.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from ._lib import Idx2Error, Params, ctx, lib, torch_ready


@dataclass(frozen=True)
class Format:
    """What D depends on: grid dims (x, y, z), dtype and number of levels (32^3 bricks, or
    32x32x1 for 2D grids)."""
    dims: Sequence[int]
    dtype: str = "float32"
    num_levels: int = 2

    def params(self) -> Params:
        d = tuple(int(x) for x in self.dims)
        bd = (32, 32, 1) if d[2] == 1 else (32, 32, 32)
        return Params(dims=d, dtype=self.dtype, brick_dims=bd, num_levels=self.num_levels, tolerance=1e-3)

    @property
    def shape(self):
        d = tuple(int(x) for x in self.dims)
        return (d[2], d[1], d[0])


def _setup(L):
    L.idx2g_coeff_count.restype = ctypes.c_longlong
    L.idx2g_synth.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.POINTER(ctypes.c_double)]
    L.idx2g_synth_adjoint.argtypes = L.idx2g_synth.argtypes
    L.idx2g_coeffs.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                               ctypes.POINTER(ctypes.c_double)]
    return L


def coeff_count(fmt: Format) -> int:
    cp = fmt.params().to_c()
    n = int(_setup(lib()).idx2g_coeff_count(ctypes.byref(cp)))
    if n < 0:
        raise Idx2Error(23, "idx2g_coeff_count: format rejected")
    return n


def _torch_dtype(fmt):
    import torch
    return torch.float32 if fmt.dtype == "float32" else torch.float64


def coefficients(ds, fmt: Format, tolerance: float = 0.0):
    """The dequantised coefficients of a Dataset (decoded at `tolerance`) as a CUDA tensor."""
    import torch
    n = coeff_count(fmt)
    c = torch.empty(n, dtype=_torch_dtype(fmt), device=torch.device("cuda", ds.device))
    p = Params(input_file=ds.params.input_file, in_dir=ds.params.in_dir, decode_tolerance=float(tolerance))
    cp = p.to_c()
    kms = ctypes.c_double(0)
    torch_ready(c.device)
    rc = _setup(lib()).idx2g_coeffs(ds._ctx.h, ds.h, ctypes.byref(cp), ctypes.c_void_p(c.data_ptr()),
                                    ctypes.c_size_t(c.numel() * c.element_size()), ctypes.byref(kms))
    if rc:
        raise Idx2Error(rc, "idx2g_coeffs")
    return c


# Kernel milliseconds of the last synth / adjoint call (CUDA events on the library's stream).
last_kernel_ms = {"synth": 0.0, "adjoint": 0.0}


def _run(fn, fmt: Format, src, nbatch: int, out):
    cp = fmt.params().to_c()
    kms = ctypes.c_double(0)
    torch_ready(src.device)
    rc = fn(ctx(src.device.index or 0).h, ctypes.byref(cp), nbatch, ctypes.c_void_p(src.data_ptr()),
            ctypes.c_void_p(out.data_ptr()), ctypes.byref(kms))
    if rc:
        raise Idx2Error(rc, "idx2g_synth")
    return kms.value


def synth(coeffs, fmt: Format):
    """grid = D(coeffs); coeffs shaped (n,) or (batch, n) on the GPU; returns (batch?, nz, ny, nx)."""
    import torch
    c = coeffs.contiguous()
    batched = c.dim() == 2
    nb = c.shape[0] if batched else 1
    if c.shape[-1] != coeff_count(fmt) or c.dtype != _torch_dtype(fmt) or not c.is_cuda:
        raise Idx2Error(101, "synth: coefficient tensor does not match the format")
    out = torch.empty((nb,) + fmt.shape, dtype=c.dtype, device=c.device)
    last_kernel_ms["synth"] = _run(_setup(lib()).idx2g_synth, fmt, c, nb, out)
    return out if batched else out[0]


def synth_adjoint(grad, fmt: Format):
    """coefficient gradient = D^T(grad); grad shaped like synth's output."""
    import torch
    g = grad.contiguous()
    batched = g.dim() == 4
    nb = g.shape[0] if batched else 1
    out = torch.empty((nb, coeff_count(fmt)), dtype=g.dtype, device=g.device)
    if g.shape[-3:] != fmt.shape or g.dtype != _torch_dtype(fmt) or not g.is_cuda:
        raise Idx2Error(101, "synth_adjoint: gradient tensor does not match the format")
    last_kernel_ms["adjoint"] = _run(_setup(lib()).idx2g_synth_adjoint, fmt, g, nb, out)
    return out if batched else out[0]


def _function():
    import torch

    class DecodeFunction(torch.autograd.Function):
        """grid = D(coefficients), with the hand-written adjoint kernel as the backward pass."""

        @staticmethod
        def forward(ctx_, coeffs, fmt):
            ctx_.fmt = fmt
            return synth(coeffs, fmt)

        @staticmethod
        def backward(ctx_, grad):
            return synth_adjoint(grad, ctx_.fmt), None

    return DecodeFunction


_FN = None


def decode_diff(coeffs, fmt: Format):
    """Differentiable decode: D(coeffs) recorded for autograd."""
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(coeffs, fmt)
