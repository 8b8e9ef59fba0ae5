"""Parsing and comparison of idx2 dataset directories (test helper).

A data file is  [bit-plane chunks][chunk sizes][i32][zstd addrs][i32][i32 n]
                [exp chunks][exp sizes][i32][zstd addrs][i32][i32 n][i32 total]
(layout written by the reference's FlushChunks / FlushChunkExponents).
Datasets are compared byte for byte, zstd frames included (the library writes the frames
the reference's vendored zstd 1.4.5 writes); where files differ, the structural parse
(decompressed frames, chunk tables) says which part.
"""
from __future__ import annotations

import ctypes
import os
import struct

_z = None


def _zstd():
    global _z
    if _z is None:
        _z = ctypes.CDLL("libzstd.so.1")
        _z.ZSTD_decompress.restype = ctypes.c_size_t
        _z.ZSTD_decompress.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t]
        _z.ZSTD_getFrameContentSize.restype = ctypes.c_ulonglong
        _z.ZSTD_getFrameContentSize.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
    return _z


def zstd_decompress(b: bytes) -> bytes:
    if len(b) == 0:
        return b""
    z = _zstd()
    n = z.ZSTD_getFrameContentSize(b, len(b))
    out = ctypes.create_string_buffer(max(n, 1))
    r = z.ZSTD_decompress(out, n, b, len(b))
    assert r == n, (r, n)
    return out.raw[:n]


def varbytes(buf: bytes):
    vals, v, sh = [], 0, 0
    for byte in buf:
        v |= (byte & 0x7F) << (7 * sh)
        sh += 1
        if not (byte & 0x80):
            vals.append(v)
            v, sh = 0, 0
    return vals


def parse_data_file(data: bytes):
    i32 = lambda off: struct.unpack("<i", data[off:off + 4])[0]
    E = len(data)
    out = {}
    total = i32(E - 4)
    nexp = i32(E - 8)
    asz = i32(E - 12)
    exp_addrs = data[E - 12 - asz:E - 12]
    ssz = i32(E - 16 - asz)
    exp_sizes = data[E - 16 - asz - ssz:E - 16 - asz]
    beg = E - total
    sizes = varbytes(exp_sizes)
    chunks, off = [], beg
    for s in sizes:
        chunks.append(zstd_decompress(data[off:off + s]))
        off += s
    out["exp_n"] = nexp
    out["exp_addrs"] = zstd_decompress(exp_addrs)
    out["exp_chunks"] = chunks
    out["exp_sizes_count"] = len(sizes)
    E2 = beg
    if E2 > 0:
        n = i32(E2 - 4)
        asz2 = i32(E2 - 8)
        addrs = data[E2 - 8 - asz2:E2 - 8]
        ssz2 = i32(E2 - 12 - asz2)
        csizes = varbytes(data[E2 - 12 - asz2 - ssz2:E2 - 12 - asz2])
        out["chunk_n"] = n
        out["chunk_addrs"] = zstd_decompress(addrs)
        out["chunk_sizes"] = csizes
        body_end = E2 - 12 - asz2 - ssz2
        out["chunk_body"] = data[:body_end]
    return out


def compare_dirs(ref_dir: str, our_dir: str):
    """Return a list of differences between two dataset directories (empty = every file
    byte-identical)."""
    diffs = []
    ref_files = sorted(os.path.relpath(os.path.join(r, f), ref_dir)
                       for r, _, fs in os.walk(ref_dir) for f in fs)
    our_files = sorted(os.path.relpath(os.path.join(r, f), our_dir)
                       for r, _, fs in os.walk(our_dir) for f in fs)
    if ref_files != our_files:
        diffs.append(("file list", ref_files, our_files))
        return diffs
    for rel in ref_files:
        a = open(os.path.join(ref_dir, rel), "rb").read()
        b = open(os.path.join(our_dir, rel), "rb").read()
        if a == b:
            continue
        if rel.endswith(".idx2"):
            sa = a.split(b"\n\n-----")[0]
            sb = b.split(b"\n\n-----")[0]
            diffs.append((rel, "metadata" if sa != sb else "statistics", sa if sa != sb else a, sb if sa != sb else b))
            continue
        pa, pb = parse_data_file(a), parse_data_file(b)
        parts = [k for k in pa if pa[k] != pb.get(k)]
        diffs.append((rel, "bytes", parts or "zstd frames (same content)"))
    return diffs
