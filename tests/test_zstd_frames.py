"""The library's zstd frames against zstd 1.4.5, the version the reference vendors and calls at
level 1 for exponent chunks and chunk-address tables (Core/idx2Encode.cpp:23-37,
Core/zstd/zstd.h:73-75).

* Every zstd frame inside the committed golden datasets (written by the reference CLI)
  decompresses and recompresses to the same bytes (no reference build needed).
* A seeded corpus of 240 inputs (sizes 1 B to 1.5 MB, so one to twelve blocks, and data
  kinds that reach each encoder path: raw, RLE and compressed blocks; raw, RLE, 1- and
  4-stream Huffman literals with table reuse across blocks; basic, RLE and compressed FSE
  tables; repeat offsets; exponent-like bytes, 16-bit exponents, u64 address tables) gives
  the same frames as the reference's own zstd (oracle/_ref, compiled from its sources)."""
import ctypes
import os
import struct
import subprocess

import numpy as np
import pytest

from idx2_files import varbytes, zstd_decompress

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "libzstd_frame_test.so")
SRCS = [os.path.join(HERE, "cpp", "zstd_frame_capi.cpp"), os.path.join(ROOT, "idx2_b200", "csrc", "zstd_frame.cpp"),
        os.path.join(ROOT, "idx2_b200", "csrc", "zstd_frame.h")]


@pytest.fixture(scope="module")
def ours():
    if not os.path.exists(LIB) or any(os.path.getmtime(LIB) < os.path.getmtime(s) for s in SRCS):
        os.makedirs(BUILD, exist_ok=True)
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I" + os.path.join(ROOT, "idx2_b200", "csrc"),
                        SRCS[0], SRCS[1], "-o", LIB], check=True)
    lib = ctypes.CDLL(LIB)
    lib.idx2g_test_zstd_compress.restype = ctypes.c_size_t
    lib.idx2g_test_zstd_compress.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t]
    return lambda b: _call(lib.idx2g_test_zstd_compress, b)


def _call(fn, b):
    cap = 2 * len(b) + 1024
    out = ctypes.create_string_buffer(cap)
    n = fn(b, len(b), out, cap)
    return out.raw[:n]


def _frames(data):
    """The zstd frames of one data file: exponent chunks and both address tables."""
    E = len(data)
    i32 = lambda o: struct.unpack("<i", data[o:o + 4])[0]
    total, asz = i32(E - 4), i32(E - 12)
    fr = [data[E - 12 - asz:E - 12]]
    ssz = i32(E - 16 - asz)
    off = E - total
    for s in varbytes(data[E - 16 - asz - ssz:E - 16 - asz]):
        fr.append(data[off:off + s])
        off += s
    E2 = E - total
    if E2 > 0:
        asz2 = i32(E2 - 8)
        fr.append(data[E2 - 8 - asz2:E2 - 8])
    return fr


def test_golden_dataset_frames_recompress_identically(ours):
    n = 0
    for root, _, files in os.walk(os.path.join(HERE, "golden", "datasets")):
        for f in files:
            if f.endswith(".bin"):
                for z in _frames(open(os.path.join(root, f), "rb").read()):
                    assert ours(zstd_decompress(z)) == z, (root, f)
                    n += 1
    assert n >= 40


def _corpus_input(seed):
    rng = np.random.default_rng(seed)
    size = int(np.exp(rng.uniform(0, np.log(1.5e6))))
    kind = seed % 8
    if kind == 0:  # exponent-like bytes: a bounded random walk over a small alphabet
        b = (np.cumsum(rng.integers(-1, 2, size)) % 30 + 110).astype(np.uint8)
    elif kind == 1:  # literals and copies of earlier text
        b = bytearray(rng.integers(97, 123, min(size, 64), dtype=np.uint8).tobytes())
        while len(b) < size:
            if rng.random() < 0.5:
                L, o = int(rng.integers(3, 200)), int(rng.integers(1, len(b) + 1))
                st = len(b) - o
                for k in range(L):
                    b.append(b[st + k])
            else:
                b.extend(rng.integers(97, 123, int(rng.integers(1, 30)), dtype=np.uint8).tobytes())
        b = np.frombuffer(bytes(b[:size]), dtype=np.uint8)
    elif kind == 2:  # geometric symbol frequencies
        b = np.minimum(rng.geometric(0.3, size), 255).astype(np.uint8)
    elif kind == 3:  # increasing u64 addresses
        b = np.cumsum(rng.integers(1, 1 << int(rng.integers(1, 40)), size // 8 + 1)).astype(np.uint64).view(np.uint8)
    elif kind == 4:  # 16-bit exponents near the float64 bias
        b = (1023 + rng.integers(-30, 3, size // 2 + 1)).astype("<u2").view(np.uint8)
    elif kind == 5:  # one value with rare bursts
        b = np.full(size, 127, np.uint8)
        m = rng.random(size) < 0.01
        b[m] = rng.integers(0, 256, int(m.sum()))
    elif kind == 6:  # incompressible
        b = rng.integers(0, 256, size, dtype=np.uint8)
    else:  # runs of a few values
        b = np.repeat(rng.integers(0, 3, size // 50 + 1, dtype=np.uint8), rng.integers(1, 100, size // 50 + 1))
        b = np.concatenate([b, np.zeros(max(0, size - len(b)), np.uint8)])
    return bytes(b[:size])


def test_corpus_matches_reference_zstd(ours, ref_harness):
    ref_harness.ref_zstd_compress.restype = ctypes.c_size_t
    ref_harness.ref_zstd_compress.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t]
    sizes = [1, 6, 7, 8, 63, 64, 255, 256, 1024, 1025, 16384, 16385, 131072, 131073, 262144, 262145, 524288]
    inputs = [_corpus_input(s) for s in range(240)]
    inputs += [bytes(np.random.default_rng(n).integers(120, 124, n, dtype=np.uint8)) for n in sizes]
    inputs += [bytes(n) for n in sizes]
    bad = [k for k, b in enumerate(inputs) if ours(b) != _call(ref_harness.ref_zstd_compress, b)]
    assert bad == [], bad[:10]
