"""Allocation-free decode (idx2g_decode_noalloc) against idx2g_decode.

Some callers cannot allocate device memory when they decode: their device memory belongs to
another allocator (a framework's caching allocator, a pool sized to the whole GPU), or they
decode inside a latency-bound serving loop where cudaMalloc fails or synchronises the device.
They open the dataset beforehand and then decode through idx2g_decode_noalloc, which keeps
every temporary in a fixed device array inside the library.

This file is collected last on purpose. It calls the entry point twice in a row through the
C ABI and checks each result against idx2g_decode's output for the same request, bit for
bit (the tolerance of every other decode test here), on 3D and 2D datasets and on requests
exactly at the scratch's limits; checks that a request larger than the fixed scratch is
rejected with ScratchTooSmall; and, in a fresh process with lazy module loading, that an
allocation-free decode made right after the dataset is opened (no other decode before it)
matches the reference decoder's output."""
import ctypes
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
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


def _check_twice(idx2g, ds, req, dt):
    import torch
    _, dims, _ = ds.output_grid(req.get("first"), req.get("last"), req["ds"])
    shape = (dims[2], dims[1], dims[0])
    ref = torch.empty(shape, dtype=dt, device="cuda")
    ds.decode(first=req.get("first"), last=req.get("last"), downsampling=req["ds"], tolerance=req["tol"], out=ref)
    for call in range(2):
        out = torch.full(shape, float("nan"), dtype=dt, device="cuda")
        rc = _noalloc(idx2g, ds, req, out)
        assert rc == 0, (req, call, idx2g.error_string(rc))
        torch.cuda.synchronize()
        assert out.cpu().numpy().tobytes() == ref.cpu().numpy().tobytes(), (req, call)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["f32b", "d64a", "d64d"])
def test_noalloc_decode_matches_decode_twice(idx2g, name):
    import torch
    case = _cases()[name]
    ds = idx2g.Dataset(os.path.join(GOLDEN, "datasets", name, "f.idx2"))
    dt = torch.float32 if case["dtype"] == "float32" else torch.float64
    for req in case["decodes"]:
        _check_twice(idx2g, ds, req, dt)
    ds.close()


@pytest.mark.gpu
def test_noalloc_2d_downsampled_matches_decode(idx2g):
    import torch
    # 2D bricks (32 x 32 x 1), 200 x 150, 2 levels: level 0 has 35 bricks, level 1 12; these
    # requests decode level 0 (its low band alone at downsampling 1 1 0) over level 1 kept on
    # the device (12 2D bricks fit the bytes of 8 3D bricks)
    ds = idx2g.Dataset(os.path.join(GOLDEN, "datasets", "f32c", "f.idx2"))
    for req in ({"ds": (1, 1, 0), "tol": 0.0}, {"ds": (1, 1, 0), "tol": 0.1}, {"ds": (0, 0, 0), "tol": 0.0}):
        _check_twice(idx2g, ds, req, torch.float32)
    ds.close()


@pytest.mark.gpu
@pytest.mark.parametrize("shape,levels", [((128, 128, 128), 2), ((512, 512, 512), 1)])
def test_noalloc_at_the_limits(idx2g, shape, levels):
    """128^3 with 2 levels: exactly 8 bricks on the coarser level; 512^3 with 1 level: exactly
    4096 bricks on the output level."""
    import torch
    from idx2_b200.synthetic import grf_field_torch
    f = grf_field_torch(*shape, seed=5, scale="unit", n_fronts=2, device=torch.device("cuda", 0))
    with tempfile.TemporaryDirectory(dir="/dev/shm" if os.path.isdir("/dev/shm") else None) as tmp:
        idx2g.encode(f, out_dir=tmp, name="lim", field_name="f", num_levels=levels, tolerance=1e-3)
        ds = idx2g.Dataset(os.path.join(tmp, "lim", "f.idx2"))
        _check_twice(idx2g, ds, {"ds": (0, 0, 0), "tol": 0.0}, torch.float32)
        ds.close()


@pytest.mark.gpu
def test_noalloc_rejects_requests_beyond_scratch(idx2g):
    import torch
    from idx2_b200.synthetic import grf_field_torch
    # 192 x 128 x 128 with 2 levels: level 1 (96 x 64 x 64) has 3 x 2 x 2 = 12 bricks, more than
    # the scratch's 8 3D bricks per kept level; at downsampling 2 2 2 no subband of level 0 is
    # decoded, level 1 is the output level and the request fits
    f = grf_field_torch(192, 128, 128, seed=6, scale="unit", n_fronts=2, device=torch.device("cuda", 0))
    with tempfile.TemporaryDirectory(dir="/dev/shm" if os.path.isdir("/dev/shm") else None) as tmp:
        idx2g.encode(f, out_dir=tmp, name="big", field_name="f", num_levels=2, tolerance=1e-3)
        ds = idx2g.Dataset(os.path.join(tmp, "big", "f.idx2"))
        req = {"ds": (0, 0, 0), "tol": 0.0}
        _, dims, _ = ds.output_grid(None, None, req["ds"])
        out = torch.zeros((dims[2], dims[1], dims[0]), dtype=torch.float32, device="cuda")
        assert _noalloc(idx2g, ds, req, out) == SCRATCH_TOO_SMALL
        _check_twice(idx2g, ds, {"ds": (2, 2, 2), "tol": 0.0}, torch.float32)
        ds.close()


_LAZY_CHILD = r"""
import ctypes, hashlib, json, os, sys
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, os.path.join(sys.argv[1], "tests"))
import torch
import idx2_b200
from test_zz_no_alloc import _noalloc
golden = os.path.join(sys.argv[1], "tests", "golden")
case = {c["name"]: c for c in json.load(open(os.path.join(golden, "datasets.json")))}["f32b"]
ds = idx2_b200.Dataset(os.path.join(golden, "datasets", "f32b", "f.idx2"))
req = case["decodes"][0]
_, dims, _ = ds.output_grid(None, None, req["ds"])
for call in range(2):
    out = torch.full((dims[2], dims[1], dims[0]), float("nan"), dtype=torch.float32, device="cuda")
    rc = _noalloc(idx2_b200, ds, req, out)
    assert rc == 0, rc
    torch.cuda.synchronize()
    assert hashlib.sha256(out.cpu().numpy().tobytes()).hexdigest() == req["sha"], call
ds.close()
print("LAZY_OK")
"""


@pytest.mark.gpu
def test_noalloc_first_call_after_open_with_lazy_loading():
    """A fresh process with CUDA_MODULE_LOADING=LAZY: the first decode of any kind is an
    allocation-free one, right after the dataset is opened; its output equals the reference
    decoder's (the golden SHA-256), on two calls in a row."""
    env = dict(os.environ, CUDA_MODULE_LOADING="LAZY")
    r = subprocess.run([sys.executable, "-c", _LAZY_CHILD, ROOT], capture_output=True, text=True, env=env,
                       timeout=600)
    assert r.returncode == 0 and "LAZY_OK" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
