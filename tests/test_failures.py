"""Failure injection on the host: data files that are missing, truncated or corrupted, and an
exponent chunk taken out of a file's chunk table.

The reference decoder reads a brick's exponents for every decoded subband before its bit
planes and fails with FileNotFound when the brick's data file is absent and with
ChunkNotFound when the file has no exponent chunk for it (Core/idx2Decode.cpp:104-106,
Core/idx2Read.cpp:270,378-388); a missing bit-plane chunk only ends that subband's planes
(Core/idx2Decode.cpp:166-168). A request that needs no brick of the damaged file decodes as
before. An exponent section whose chunk count does not match its size list, or is not a
whole number of subband sets, fails with SizeMismatched (Core/idx2Read.cpp:316-323). The CPU
tests pin these codes on the reference CLI (oracle/_ref); the GPU tests check
this library's decoder on the same damaged datasets: the same codes, and for damage the
reference does not detect (a truncated file, chunk sizes beyond the file) CorruptStream at
open instead of a read past the data. Nothing here touches the GPU's memory or state: every
failure is made in the files, on the host."""
import ctypes
import hashlib
import json
import os
import shutil
import struct
import subprocess
import tempfile

import pytest

from idx2_files import varbytes, zstd_decompress

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def _case(name):
    return {c["name"]: c for c in json.load(open(os.path.join(GOLDEN, "datasets.json")))}[name]


def _zstd_compress(b: bytes) -> bytes:
    z = ctypes.CDLL("libzstd.so.1")
    z.ZSTD_compressBound.restype = ctypes.c_size_t
    z.ZSTD_compress.restype = ctypes.c_size_t
    z.ZSTD_compress.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    cap = z.ZSTD_compressBound(ctypes.c_size_t(len(b)))
    out = ctypes.create_string_buffer(cap)
    n = z.ZSTD_compress(out, cap, b, len(b), 1)
    return out.raw[:n]


def _varbyte(v: int) -> bytes:
    out = bytearray()
    while True:
        b = v & 0x7F
        v >>= 7
        if v:
            out.append(b | 0x80)
        else:
            out.append(b)
            return bytes(out)


def _edit_exponent_chunks(path: str, k: int, drop: bool):
    """Rewrite a data file's exponent section: drop its k-th exponent chunk (bytes, size and
    address), or keep the chunk and give it the address of a chunk that does not exist."""
    data = open(path, "rb").read()
    E = len(data)
    i32 = lambda off: struct.unpack("<i", data[off:off + 4])[0]
    total, nexp, asz = i32(E - 4), i32(E - 8), i32(E - 12)
    addrs = zstd_decompress(data[E - 12 - asz:E - 12])
    ssz = i32(E - 16 - asz)
    sizes = varbytes(data[E - 16 - asz - ssz:E - 16 - asz])
    beg = E - total
    chunks, off = [], beg
    for s in sizes:
        chunks.append(data[off:off + s])
        off += s
    assert 0 <= k < nexp == len(sizes)
    if drop:
        del chunks[k], sizes[k]
        addrs = addrs[:8 * k] + addrs[8 * k + 8:]
    else:
        a = struct.unpack("<Q", addrs[8 * k:8 * k + 8])[0] + (4093 << 18)  # another chunk index
        addrs = addrs[:8 * k] + struct.pack("<Q", a) + addrs[8 * k + 8:]
    za = _zstd_compress(addrs)
    vb = b"".join(_varbyte(s) for s in sizes)
    sec = b"".join(chunks) + vb + struct.pack("<i", len(vb)) + za + struct.pack("<i", len(za)) + \
        struct.pack("<i", len(sizes))
    sec += struct.pack("<i", len(sec) + 4)
    open(path, "wb").write(data[:beg] + sec)


def _damaged(tmp, name, how):
    """A copy of golden dataset `name` under tmp with one kind of damage; returns the .idx2 path."""
    src = os.path.join(GOLDEN, "datasets", name)
    dst = os.path.join(tmp, name)
    shutil.copytree(src, dst)
    f0 = os.path.join(dst, "f", "L00.bin")
    if how == "missing_L00":
        os.remove(f0)
    elif how == "missing_L01":
        os.remove(os.path.join(dst, "f", "L01.bin"))
    elif how == "no_exponent_chunk":
        _edit_exponent_chunks(f0, 0, drop=False)
    elif how == "exponent_chunk_dropped":
        _edit_exponent_chunks(f0, 0, drop=True)
    elif how == "truncated":
        data = open(f0, "rb").read()
        open(f0, "wb").write(data[:len(data) - 9])
    elif how == "chunk_sizes_past_end":
        # the first varbyte of the bit-plane chunk sizes made to claim more bytes than the file
        data = bytearray(open(f0, "rb").read())
        E = len(data)
        i32 = lambda off: struct.unpack("<i", bytes(data[off:off + 4]))[0]
        E2 = E - i32(E - 4)
        asz2 = i32(E2 - 8)
        ssz2 = i32(E2 - 12 - asz2)
        p = E2 - 12 - asz2 - ssz2
        data[p] |= 0x7F  # (the low 7 bits of the first chunk's size)
        data[p + 1] = (data[p + 1] | 0x7F) if (data[p] & 0x80) else data[p + 1]
        open(f0, "wb").write(bytes(data))
    return os.path.join(dst, "f.idx2")


def _ref_decode(ref_app, idx2_path, out_dir, ds=(0, 0, 0)):
    r = subprocess.run([ref_app, "--decode", idx2_path, "--downsampling", *map(str, ds), "--out_dir", out_dir,
                        "--out_file", "o.raw"], capture_output=True, text=True, timeout=300)
    out = None
    if r.returncode == 0:
        out = open(os.path.join(out_dir, "o.raw"), "rb").read()
    return r.returncode, r.stdout + r.stderr, out


# ----------------------------------------------------------------------------------------------
# the reference's behaviour (CPU)

FAILURES = [("missing_L00", "FileNotFound"), ("no_exponent_chunk", "ChunkNotFound"),
            ("exponent_chunk_dropped", "SizeMismatched")]


@pytest.mark.parametrize("how,code", FAILURES)
def test_reference_decode_fails_with(ref_app, how, code):
    with tempfile.TemporaryDirectory() as tmp:
        p = _damaged(tmp, "f32b", how)
        rc, msg, _ = _ref_decode(ref_app, p, tmp)
        if code == "ChunkNotFound":
            # the reference's ReadChunkExponents returns ChunkNotFound (Core/idx2Read.cpp:388), and
            # the CLI then dies with a segmentation fault on the way out (measured here)
            assert rc != 0, (rc, msg[-500:])
        else:
            assert rc != 0 and code in msg, (rc, msg[-500:])


def test_reference_decode_skips_an_unused_missing_file(ref_app):
    # at downsampling 1 1 1 the 2-level dataset decodes level 1 only: L00.bin is not read
    case = _case("f32b")
    want = [d for d in case["decodes"] if d["ds"] == [1, 1, 1] and d["tol"] == 0.0][0]
    with tempfile.TemporaryDirectory() as tmp:
        p = _damaged(tmp, "f32b", "missing_L00")
        rc, msg, out = _ref_decode(ref_app, p, tmp, ds=(1, 1, 1))
        assert rc == 0, msg[-500:]
        assert hashlib.sha256(out).hexdigest() == want["sha"]


def test_reference_decode_of_a_truncated_file_fails(ref_app):
    with tempfile.TemporaryDirectory() as tmp:
        p = _damaged(tmp, "f32b", "truncated")
        rc, msg, _ = _ref_decode(ref_app, p, tmp)
        assert rc != 0, msg[-500:]


# ----------------------------------------------------------------------------------------------
# this library (GPU)

def _open(idx2g, path):
    return idx2g.Dataset(path)


@pytest.mark.gpu
@pytest.mark.parametrize("how,code", FAILURES)
def test_decode_fails_with_the_reference_code(idx2g, how, code):
    with tempfile.TemporaryDirectory() as tmp:
        ds = _open(idx2g, _damaged(tmp, "f32b", how))
        with pytest.raises(idx2g.Idx2Error) as ei:
            ds.decode()
        assert idx2g.error_string(ei.value.code) == code
        ds.close()


@pytest.mark.gpu
def test_decode_skips_an_unused_missing_file(idx2g):
    case = _case("f32b")
    want = [d for d in case["decodes"] if d["ds"] == [1, 1, 1] and d["tol"] == 0.0][0]
    with tempfile.TemporaryDirectory() as tmp:
        ds = _open(idx2g, _damaged(tmp, "f32b", "missing_L00"))
        out = ds.decode(downsampling=(1, 1, 1))
        ds.close()
    assert hashlib.sha256(out.tobytes()).hexdigest() == want["sha"]


@pytest.mark.gpu
@pytest.mark.parametrize("how", ["truncated", "chunk_sizes_past_end"])
def test_open_rejects_a_corrupt_file(idx2g, how):
    with tempfile.TemporaryDirectory() as tmp:
        with pytest.raises(idx2g.Idx2Error) as ei:
            _open(idx2g, _damaged(tmp, "f32b", how))
        assert idx2g.error_string(ei.value.code) == "CorruptStream"
