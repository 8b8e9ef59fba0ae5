"""Decode side of the Python mirror: idx2::Init / GetOutputGrid / Decode / Destroy
(idx2.cpp:23-52) over the C ABI."""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

from ._lib import Idx2Error, Params, _CParams, ctx, lib, torch_ready


class Dataset:
    """A compressed dataset made resident on the device (idx2g_dataset_open)."""

    def __init__(self, idx2_file: str, in_dir: Optional[str] = None, device: int = 0):
        if in_dir is None:
            # the CLI's rule: the directory two levels above the .idx2 file
            parent = os.path.dirname(idx2_file)
            in_dir = os.path.dirname(parent) or "."
            if in_dir == parent:
                in_dir = "./"
        self.device = device
        self.params = Params(input_file=idx2_file, in_dir=in_dir)
        self._ctx = ctx(device)
        h = ctypes.c_void_p()
        cp = self.params.to_c()
        rc = lib().idx2g_dataset_open(self._ctx.h, ctypes.byref(cp), ctypes.byref(h))
        if rc:
            raise Idx2Error(rc, "idx2g_dataset_open")
        self.h = h
        name, field = ctypes.create_string_buffer(64), ctypes.create_string_buffer(64)
        dims, dt, nl = (ctypes.c_int * 3)(), ctypes.c_int(), ctypes.c_int()
        tol, res = ctypes.c_double(), ctypes.c_longlong()
        rc = lib().idx2g_dataset_info(h, name, field, dims, ctypes.byref(dt), ctypes.byref(nl), ctypes.byref(tol),
                                      ctypes.byref(res))
        if rc:
            raise Idx2Error(rc, "idx2g_dataset_info")
        self._dtype = np.float32 if dt.value == 0 else np.float64  # IDX2G_FLOAT32 = 0
        self.dims = tuple(dims)
        self.num_levels = nl.value
        self.tolerance = tol.value
        self.resident_bytes = res.value

    def _req(self, first, last, downsampling, tolerance) -> Params:
        p = Params(input_file=self.params.input_file, in_dir=self.params.in_dir,
                   downsampling=tuple(downsampling), decode_tolerance=float(tolerance))
        if first is not None:
            p.first, p.last = tuple(first), tuple(last)
        return p

    def output_grid(self, first=None, last=None, downsampling=(0, 0, 0)):
        p = self._req(first, last, downsampling, 0.0)
        f, d, s = (ctypes.c_int * 3)(), (ctypes.c_int * 3)(), (ctypes.c_int * 3)()
        cp = p.to_c()
        rc = lib().idx2g_output_grid(self.h, ctypes.byref(cp), f, d, s)
        if rc:
            raise Idx2Error(rc, "idx2g_output_grid")
        return tuple(f), tuple(d), tuple(s)

    def decode(self, first: Optional[Sequence[int]] = None, last: Optional[Sequence[int]] = None,
               downsampling=(0, 0, 0), tolerance: float = 0.0, out=None, dtype=None):
        """Decode to a numpy array (or into `out`: numpy array or CUDA torch tensor) shaped
        (nz, ny, nx) of the output grid."""
        _, dims, _ = self.output_grid(first, last, downsampling)
        p = self._req(first, last, downsampling, tolerance)
        cp = p.to_c()
        if out is None:
            out = np.zeros((dims[2], dims[1], dims[0]), dtype=dtype or self.dtype)
        on_dev = 0
        try:
            import torch
            if isinstance(out, torch.Tensor):
                on_dev = int(out.is_cuda)
                ptr, nbytes = out.data_ptr(), out.numel() * out.element_size()
            else:
                ptr, nbytes = out.ctypes.data, out.nbytes
        except ImportError:
            ptr, nbytes = out.ctypes.data, out.nbytes
        if on_dev:
            torch_ready(out.device)
        kms = ctypes.c_double(0)
        rc = lib().idx2g_decode(self._ctx.h, self.h, ctypes.byref(cp), ctypes.c_void_p(ptr),
                                ctypes.c_size_t(nbytes), on_dev, ctypes.byref(kms))
        if rc:
            raise Idx2Error(rc, "idx2g_decode")
        self.last_kernel_ms = kms.value
        return out

    def decode_batch(self, requests, device_out: bool = True):
        """Decode several requests in one call (idx2g_decode_batch): requests is a list of dicts
        with optional keys first, last, downsampling, tolerance (as in decode). Returns one
        array per request: CUDA torch tensors when device_out, numpy arrays otherwise."""
        n = len(requests)
        if n == 0:
            return []
        cps = (_CParams * n)()
        outs, ptrs, sizes, shapes = [], [], [], []
        dt = self.dtype
        esz = np.dtype(dt).itemsize
        import torch
        for i, r in enumerate(requests):
            first, last = r.get("first"), r.get("last")
            ds = r.get("downsampling", (0, 0, 0))
            p = self._req(first, last, ds, r.get("tolerance", 0.0))
            cps[i] = p.to_c()
            _, dims, _ = self.output_grid(first, last, ds)
            shapes.append((dims[2], dims[1], dims[0]))
            sizes.append(int(np.prod(shapes[-1])) * esz)
        if device_out:
            # one allocation for the whole call (each grid 256-byte aligned), the grids are views
            # of it: a serving loop of varying batches then reuses a few cached blocks
            offs, total = [], 0
            for b in sizes:
                offs.append(total)
                total += (b + 255) & ~255
            arena = torch.empty(max(total, 1), dtype=torch.uint8, device=torch.device("cuda", self.device))
            tdt = torch.float32 if dt == np.float32 else torch.float64
            for shape, off, b in zip(shapes, offs, sizes):
                o = arena[off:off + b].view(tdt).view(shape)
                outs.append(o)
                ptrs.append(arena.data_ptr() + off)
        else:
            for shape in shapes:
                o = np.empty(shape, dtype=dt)
                outs.append(o)
                ptrs.append(o.ctypes.data)
        arr = (ctypes.c_void_p * n)(*[ctypes.c_void_p(q) for q in ptrs])
        szs = (ctypes.c_size_t * n)(*sizes)
        kms = ctypes.c_double(0)
        L = lib()
        L.idx2g_decode_batch.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(_CParams), ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_double)]
        if device_out:
            torch_ready(torch.device("cuda", self.device))
        rc = L.idx2g_decode_batch(self._ctx.h, self.h, cps, n, arr, szs, int(device_out), ctypes.byref(kms))
        if rc:
            raise Idx2Error(rc, "idx2g_decode_batch")
        self.last_kernel_ms = kms.value
        return outs

    def decode_brick_map(self, path: str, downsampling=(0, 0, 0), tolerance: float = 0.0):
        """The reference's HashMap output mode (idx2App --brick_map): every finest brick at
        the finest resolution that is significant for it, written to `path` in the reference's
        bricks-file layout (idx2g_decode_brick_map)."""
        p = self._req(None, None, downsampling, tolerance)
        cp = p.to_c()
        kms = ctypes.c_double(0)
        L = lib()
        L.idx2g_decode_brick_map.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(_CParams),
                                             ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)]
        rc = L.idx2g_decode_brick_map(self._ctx.h, self.h, ctypes.byref(cp), os.fsencode(path), ctypes.byref(kms))
        if rc:
            raise Idx2Error(rc, "idx2g_decode_brick_map")
        self.last_kernel_ms = kms.value
        return path

    @property
    def dtype(self):
        return self._dtype

    def close(self):
        if getattr(self, "h", None):
            lib().idx2g_dataset_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
