"""Sharded encode on the CPU: world_size 2 (and 3) torch.distributed gloo ranks each code the
subtrees of their run of coarsest bricks (the oracle's brick coder standing in for the GPU),
exchange their region headers with all_gather, reduce the value range with all_reduce, and
write their parts of one dataset. The files are compared byte for byte with the
single-process encode of the same field (the library's plan and packer with the same coder)
and, where the reference CLI is built, with the reference's own encode."""
import ctypes
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from idx2_files import compare_dirs
from oracle_tools import oracle_encode

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle_shard.so")
CSRC = os.path.join(ROOT, "idx2_b200", "csrc")
SRCS = [os.path.join(HERE, "cpp", "oracle_shard.cpp")] + [os.path.join(CSRC, f) for f in (
    "format.cpp", "packer.cpp", "encoder.cpp", "shard.cpp", "zstd_frame.cpp")]
DEPS = SRCS + [os.path.join(HERE, "cpp", "oracle_coder.h"), os.path.join(CSRC, "shard.h"),
               os.path.join(CSRC, "packer.h"), os.path.join(CSRC, "encoder.h"),
               os.path.join(ROOT, "oracle", "idx2_oracle.c")]


def build_lib():
    if os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in DEPS):
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    obj = os.path.join(BUILD, "idx2_oracle_pic.o")
    subprocess.run(["gcc", "-O2", "-std=c11", "-fPIC", "-ffp-contract=off", "-c",
                    os.path.join(ROOT, "oracle", "idx2_oracle.c"), "-o", obj], check=True)
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-I" + CSRC,
                    "-I" + os.path.join(ROOT, "oracle")] + SRCS + [obj, "-o", LIB, "-ldl", "-lm"], check=True)
    return LIB


def _rank_main(rank, world, port, raw, dims, f32, levels, tol, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        L = ctypes.CDLL(LIB)
        L.oshard_begin.restype = ctypes.c_void_p
        L.oshard_begin.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_double, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                   ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.oshard_headers.restype = ctypes.c_size_t
        L.oshard_headers.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
        L.oshard_range.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
        L.oshard_finish.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                    ctypes.c_double]
        L.oshard_free.argtypes = [ctypes.c_void_p]
        err = ctypes.c_int(0)
        h = L.oshard_begin(raw.encode(), dims[0], dims[1], dims[2], int(f32), levels, tol, out_dir.encode(),
                           b"shd", b"f", rank, world, ctypes.byref(err))
        assert h and err.value == 0, err.value
        p = ctypes.c_void_p()
        n = L.oshard_headers(h, ctypes.byref(p))
        mine = torch.frombuffer(bytearray(ctypes.string_at(p, n)), dtype=torch.uint8) if n else torch.zeros(0, dtype=torch.uint8)
        # the exchange: payload sizes, then the payloads padded to the largest
        sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(sizes, torch.tensor([n], dtype=torch.int64))
        cap = max(int(s) for s in sizes)
        padded = torch.zeros(cap, dtype=torch.uint8)
        padded[:n] = mine
        parts = [torch.zeros(cap, dtype=torch.uint8) for _ in range(world)]
        dist.all_gather(parts, padded)
        lo, hi = ctypes.c_double(), ctypes.c_double()
        L.oshard_range(h, ctypes.byref(lo), ctypes.byref(hi))
        rng = torch.tensor([-lo.value, hi.value], dtype=torch.float64)
        dist.all_reduce(rng, op=dist.ReduceOp.MAX)
        keep = [bytes(parts[s][:int(sizes[s])].numpy()) for s in range(world)]
        ptrs = (ctypes.c_void_p * world)(*[ctypes.cast(ctypes.c_char_p(b), ctypes.c_void_p) for b in keep])
        szs = (ctypes.c_size_t * world)(*[len(b) for b in keep])
        rc = L.oshard_finish(h, ptrs, szs, -float(rng[0]), float(rng[1]))
        assert rc == 0, rc
        L.oshard_free(h)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


CASES = [
    # dims, float32, levels, tol, ranks
    ((160, 128, 96), True, 2, 1e-3, 2),
    ((130, 100, 70), False, 2, 1e-4, 2),
    ((256, 256, 1), True, 3, 1e-3, 3),
    ((200, 150, 1), False, 2, 1e-3, 2),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{'f32' if c[1] else 'f64'}-L{c[2]}-r{c[4]}")
def test_sharded_encode_matches_single_encode(tmp_path, case, ref_app):
    dims, f32, levels, tol, world = case
    build_lib()
    from idx2_b200.synthetic import bumps_field
    nx, ny, nz = dims
    f = bumps_field(nx, ny, nz, seed=41).astype(np.float32 if f32 else np.float64)
    dt = "Float32" if f32 else "Float64"
    raw = str(tmp_path / f"shd-f-[{nx}-{ny}-{nz}]-{dt}.raw")
    f.tofile(raw)
    out = str(tmp_path / "sharded")
    mp.start_processes(_rank_main, args=(world, _free_port(), raw, dims, f32, levels, tol, out),
                       nprocs=world, start_method="spawn", join=True)
    # the same field through one process
    rc, err = oracle_encode(raw, dims, "float32" if f32 else "float64", levels, tol, str(tmp_path / "single"),
                            name="shd", field="f", brick=(32, 32, 1) if nz == 1 else (32, 32, 32))
    assert rc == 0, err
    assert compare_dirs(str(tmp_path / "single" / "shd"), os.path.join(out, "shd")) == []
    # and through the reference
    args = [ref_app, "--encode", raw, "--num_levels", str(levels), "--tolerance", repr(tol), "--out_dir",
            str(tmp_path / "ref")]
    if nz == 1:
        args += ["--brick_size", "32", "32", "1"]
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-300:] + r.stderr[-300:]
    assert compare_dirs(str(tmp_path / "ref" / "shd"), os.path.join(out, "shd")) == []
