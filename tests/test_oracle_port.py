"""The C restatement (oracle/) against the golden vectors made by the compiled
reference (tests/golden/kats.json, tests/golden/make_golden.py)."""
import ctypes as C
import hashlib
import json
import os

import numpy as np
import pytest

from golden.golden_inputs import brick_cases, block_cases, make_block, make_brick

HERE = os.path.dirname(os.path.abspath(__file__))
KATS = json.load(open(os.path.join(HERE, "golden", "kats.json")))


def sha(b):
    return hashlib.sha256(b).hexdigest()


def dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def up(a):
    return a.ctypes.data_as(C.POINTER(C.c_ulonglong))


def test_brick_transforms(oracle_lib):
    assert len(KATS["bricks"]) == len(brick_cases())
    for case, gold in zip(brick_cases(), KATS["bricks"]):
        b = make_brick(case)
        valid = np.array(case["valid"], np.int32)
        fwd = b.copy()
        oracle_lib.oracle_brick_forward(dp(fwd), case["is2d"], ip(valid), case["level"], case["coarsest"])
        assert sha(fwd.tobytes()) == gold["forward"], case
        ext = b.copy()
        oracle_lib.oracle_brick_extrapolate(dp(ext), case["is2d"], ip(valid))
        assert sha(ext.tobytes()) == gold["extrapolate"], case
        inv = fwd.copy()
        oracle_lib.oracle_brick_inverse(dp(inv), case["is2d"], case["level"], case["coarsest"])
        assert sha(inv.tobytes()) == gold["inverse"], case


def test_block_coder(oracle_lib):
    for case, gold in zip(block_cases(), KATS["blocks"]):
        vals = make_block(case)
        nd = case["ndims"]
        nv = 1 << (2 * nd)
        em = np.zeros(1, np.int32)
        uc = np.zeros(64, np.uint64)
        pb = np.zeros(64, np.int32)
        pn = np.zeros(64, np.int32)
        pbits = np.zeros(64, np.int32)
        pw = np.zeros(256, np.uint64)
        k = oracle_lib.oracle_block_encode(dp(vals), nd, case["is_f32"], C.c_double(case["tol"]), 1, ip(em),
                                           up(uc), ip(pb), ip(pn), ip(pbits), up(pw))
        assert k == gold["nplanes"] and em[0] == gold["emax"], case
        assert sha(uc[:nv].tobytes()) == gold["ucoeffs"], case
        assert pb[:k].tolist() == gold["planes"] and pn[:k].tolist() == gold["nin"], case
        assert pbits[:k].tolist() == gold["bits"], case
        assert sha(pw[:4 * k].tobytes()) == gold["words"], case
        dec = np.zeros(nv)
        if k > 0:
            oracle_lib.oracle_block_decode(nd, int(em[0]), int(k), ip(pb), up(pw), dp(dec))
        assert sha(dec.tobytes()) == gold["decoded"], case


def test_varints(oracle_lib):
    oracle_lib.oracle_varint_stream.restype = C.c_longlong
    for g in KATS["varints"]:
        vals = np.array(g["vals"], dtype=np.uint64)
        buf = np.zeros(4096, np.uint8)
        nbits = oracle_lib.oracle_varint_stream(up(vals), g["n_var"], len(vals), buf.ctypes.data_as(C.c_char_p),
                                                C.c_longlong(4096))
        assert nbits == g["nbits"]
        assert buf[:(nbits + 7) // 8].tobytes().hex() == g["bytes"]


@pytest.mark.parametrize("xyz", [(0, 0, 0), (1, 2, 3), (7, 5, 1), (4, 4, 4), (1023, 0, 512)])
def test_morton(oracle_lib, xyz):
    oracle_lib.oracle_encode_morton3.restype = C.c_uint32
    x, y, z = xyz
    expect = 0
    for i in range(10):
        expect |= ((x >> i) & 1) << (3 * i) | ((y >> i) & 1) << (3 * i + 1) | ((z >> i) & 1) << (3 * i + 2)
    assert oracle_lib.oracle_encode_morton3(x, y, z) == expect


def test_oracle_matches_live_reference(oracle_lib, ref_harness):
    """Fresh random bricks (not in the fixtures) through both, when the reference is built."""
    rng = np.random.default_rng(77)
    for t in range(6):
        valid = [int(rng.integers(1, 33)) for _ in range(3)]
        b = np.zeros((33, 33, 33))
        b[:valid[2], :valid[1], :valid[0]] = rng.normal(size=valid[::-1])
        r, o = b.copy(), b.copy()
        ref_harness.ref_brick_forward(dp(r), 32, *valid, 1, 0)
        oracle_lib.oracle_brick_forward(dp(o), 0, ip(np.array(valid, np.int32)), 1, 0)
        assert r.tobytes() == o.tobytes()
