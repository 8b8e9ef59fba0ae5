"""One field encoded by several processes, one GPU each, into one dataset (idx2g_encode_shard).

The split follows the reference's depth-first encode (Core/idx2Encode.cpp:276-340): the
coarsest level's bricks, in encode order, are cut into one run per process, and each process
codes the subtrees under its run from the samples of its region (`shard_region`). The coded
data never moves: the processes all-gather the headers of their (brick, subband) regions and
all-reduce the value range through torch.distributed (NCCL or gloo), then each writes its
own bytes into the shared dataset files. The files equal a single-process encode's.

    >>> dist.init_process_group("nccl")
    >>> lo, dims = shard_region(global_dims, "float32", 3, 1e-3, rank, world)
    >>> info = encode_sharded(local_field, lo, global_dims, out_dir, "grf", "f", 3, 1e-3)
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from ._lib import EncodeInfo, Idx2Error, Params, _CParams, _Ctx, _field_ptr, ctx, lib, torch_ready


def _params(dims, dtype, num_levels, tolerance, out_dir=".", name="field", field_name="data"):
    bd = (32, 32, 1) if dims[2] == 1 else (32, 32, 32)
    return Params(name=name, field=field_name, dims=tuple(dims), dtype=dtype, brick_dims=bd,
                  num_levels=num_levels, tolerance=tolerance, out_dir=out_dir)


def _bind():
    L = lib()
    if getattr(L, "_shard_bound", False):
        return L
    L.idx2g_shard_region.argtypes = [ctypes.POINTER(_CParams), ctypes.c_int, ctypes.c_int, ctypes.c_int * 3,
                                     ctypes.c_int * 3]
    L.idx2g_encode_shard.argtypes = [ctypes.c_void_p, ctypes.POINTER(_CParams), ctypes.c_void_p, ctypes.c_int * 3,
                                     ctypes.c_int * 3, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_void_p),
                                     ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_double),
                                     ctypes.POINTER(ctypes.c_double), ctypes.POINTER(EncodeInfo)]
    L.idx2g_encode_shard_finish.argtypes = [ctypes.c_void_p, ctypes.POINTER(_CParams), ctypes.c_int, ctypes.c_int,
                                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                            ctypes.POINTER(EncodeInfo)]
    L._shard_bound = True
    return L


def shard_region(dims: Sequence[int], dtype: str, num_levels: int, tolerance: float, shard: int, nshards: int):
    """(first, size) of the samples shard `shard` of `nshards` reads, each (x, y, z)."""
    cp = _params(dims, dtype, num_levels, tolerance).to_c()
    lo, n = (ctypes.c_int * 3)(), (ctypes.c_int * 3)()
    rc = _bind().idx2g_shard_region(ctypes.byref(cp), shard, nshards, lo, n)
    if rc:
        raise Idx2Error(rc, "idx2g_shard_region")
    return tuple(lo), tuple(n)


class ShardEncode:
    """The two halves of one shard's encode on one context: code (begin), then, with every
    shard's header payload, write (finish). For callers that exchange the payloads themselves.
    A context holds one shard's coded state between the halves: shards whose halves interleave
    in one process need a context each (`own_context`)."""

    def __init__(self, field, origin, dims, out_dir, name, field_name, num_levels, tolerance, shard, nshards,
                 device: int = 0, device_only: bool = False, own_context: bool = False):
        ptr, on_dev, dt, ldims, self._keep = _field_ptr(field)
        if not on_dev:
            raise Idx2Error(101, "a shard's field must be a CUDA tensor")
        self.shard, self.nshards = shard, nshards
        self._cp = _params(dims, dt, num_levels, tolerance, out_dir, name, field_name).to_c()
        self._ctx = _Ctx(device) if own_context else ctx(device)
        self.info = EncodeInfo()
        hp, hn = ctypes.c_void_p(), ctypes.c_size_t()
        lo, hi = ctypes.c_double(), ctypes.c_double()
        torch_ready(self._keep.device)
        rc = _bind().idx2g_encode_shard(self._ctx.h, ctypes.byref(self._cp), ctypes.c_void_p(ptr),
                                        (ctypes.c_int * 3)(*origin), (ctypes.c_int * 3)(*ldims), shard, nshards,
                                        1 if device_only else 0, ctypes.byref(hp), ctypes.byref(hn),
                                        ctypes.byref(lo), ctypes.byref(hi),
                                        ctypes.byref(self.info))
        if rc:
            raise Idx2Error(rc, "idx2g_encode_shard")
        self.headers = ctypes.string_at(hp, hn.value) if hn.value else b""
        self.vmin, self.vmax = lo.value, hi.value

    def finish(self, payloads: Sequence[bytes], vmin: float, vmax: float) -> EncodeInfo:
        n = self.nshards
        keep = [bytes(b) for b in payloads]
        ptrs = (ctypes.c_void_p * n)(*[ctypes.cast(ctypes.c_char_p(b), ctypes.c_void_p) for b in keep])
        sizes = (ctypes.c_size_t * n)(*[len(b) for b in keep])
        rc = _bind().idx2g_encode_shard_finish(self._ctx.h, ctypes.byref(self._cp), self.shard, n, ptrs, sizes,
                                               vmin, vmax, ctypes.byref(self.info))
        self._keep = None
        if rc:
            raise Idx2Error(rc, "idx2g_encode_shard_finish")
        return self.info


def exchange(payload: bytes, vmin: float, vmax: float, group=None):
    """All-gather the header payloads and all-reduce the value range over the process group
    (NCCL groups exchange device tensors, others host tensors). Returns (payloads, vmin, vmax)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")
    n = len(payload)
    sizes = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(sizes, torch.tensor([n], dtype=torch.int64, device=dev), group=group)
    cap = max(int(s) for s in sizes)
    mine = torch.zeros(max(cap, 1), dtype=torch.uint8)
    if n:
        mine[:n] = torch.frombuffer(bytearray(payload), dtype=torch.uint8)
    mine = mine.to(dev)
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    rng = torch.tensor([-vmin, vmax], dtype=torch.float64, device=dev)
    dist.all_reduce(rng, op=dist.ReduceOp.MAX, group=group)
    rng = rng.cpu()
    out = [bytes(parts[s][:int(sizes[s])].cpu().numpy()) for s in range(world)]
    return out, -float(rng[0]), float(rng[1])


def encode_sharded(field, origin: Sequence[int], dims: Sequence[int], out_dir: str, name: str, field_name: str,
                   num_levels: int, tolerance: float, group=None, device: Optional[int] = None) -> EncodeInfo:
    """This process's shard of one encode (rank and world size of the process group): field
    (CUDA tensor, shape (nz, ny, nx)) holds the dataset's samples [origin, origin + its dims),
    covering at least shard_region(...) of this rank. Returns when this shard's bytes are
    written; the dataset is complete after a barrier of the group."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    dev = field.device.index if device is None else device
    job = ShardEncode(field, origin, dims, out_dir, name, field_name, num_levels, tolerance, rank, world, dev)
    payloads, vmin, vmax = exchange(job.headers, job.vmin, job.vmax, group)
    info = job.finish(payloads, vmin, vmax)
    dist.barrier(group)
    return info
