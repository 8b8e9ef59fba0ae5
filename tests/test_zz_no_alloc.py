"""Allocation-free decode (idx2g_decode_noalloc) against idx2g_decode.

Some callers cannot allocate device memory when they decode: their device memory belongs to
another allocator (a framework's caching allocator, a pool sized to the whole GPU), or they
decode inside a latency-bound serving loop where cudaMalloc fails or synchronises the device.
They open the dataset beforehand and then decode through idx2g_decode_noalloc, which keeps
every temporary in a fixed device array inside the library.

This file is collected last on purpose. It calls the entry point twice in a row through the
C ABI and checks each result against idx2g_decode's output for the same request, bit for
bit (the tolerance of every other decode test here), and checks that a request larger than
the fixed scratch is rejected with ScratchTooSmall."""
import ctypes
import json
import os

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
SCRATCH_TOO_SMALL = 104


def _cases():
    return {c["name"]: c for c in json.load(open(os.path.join(GOLDEN, "datasets.json")))}


def _noalloc(idx2g, ds, req, out):
    from idx2_b200 import _lib
    L = _lib.lib()
    L.idx2g_decode_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(_lib._CParams),
                                       ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_double)]
    p = ds._req(req.get("first"), req.get("last"), req["ds"], req["tol"]).to_c()
    kms = ctypes.c_double(0)
    return L.idx2g_decode_noalloc(ds._ctx.h, ds.h, ctypes.byref(p), ctypes.c_void_p(out.data_ptr()),
                                  ctypes.c_size_t(out.numel() * out.element_size()), ctypes.byref(kms))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["f32b", "d64a", "d64d"])
def test_noalloc_decode_matches_decode_twice(idx2g, name):
    import torch
    case = _cases()[name]
    ds = idx2g.Dataset(os.path.join(GOLDEN, "datasets", name, "f.idx2"))
    dt = torch.float32 if case["dtype"] == "float32" else torch.float64
    for req in case["decodes"]:
        _, dims, _ = ds.output_grid(req.get("first"), req.get("last"), req["ds"])
        shape = (dims[2], dims[1], dims[0])
        ref = torch.empty(shape, dtype=dt, device="cuda")
        ds.decode(first=req.get("first"), last=req.get("last"), downsampling=req["ds"], tolerance=req["tol"],
                  out=ref)
        for call in range(2):
            out = torch.full(shape, float("nan"), dtype=dt, device="cuda")
            rc = _noalloc(idx2g, ds, req, out)
            assert rc == 0, (req, call, idx2g.error_string(rc))
            torch.cuda.synchronize()
            assert out.cpu().numpy().tobytes() == ref.cpu().numpy().tobytes(), (req, call)
    ds.close()


@pytest.mark.gpu
def test_noalloc_rejects_requests_beyond_scratch(idx2g):
    import torch
    # the 2D golden dataset has 12 bricks on level 1, more than the scratch's 8
    ds = idx2g.Dataset(os.path.join(GOLDEN, "datasets", "f32c", "f.idx2"))
    req = {"ds": (0, 0, 0), "tol": 0.0}
    _, dims, _ = ds.output_grid(None, None, req["ds"])
    out = torch.zeros((dims[2], dims[1], dims[0]), dtype=torch.float32, device="cuda")
    assert _noalloc(idx2g, ds, req, out) == SCRATCH_TOO_SMALL
    ds.close()
