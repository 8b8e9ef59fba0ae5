"""The headline workload at full size against the reference: a 1024^3 float32 k^-5/3 Gaussian
random field (seeded, unit variance) with 20 tanh fronts, 3 levels, 32^3 bricks.

* Tolerance 1e-3 (the headline encode): the reference CLI encodes the same field from a raw
  file; this library's files equal its files (32,768 level-0 bricks in 8 chunks per channel,
  so the chunks the reference flushes in the middle of the encode, Core/idx2Encode.cpp:233-249,
  Core/idx2Write.cpp:317-386, are compared at this size). The full-resolution decode equals
  the reference's decode of the same files byte for byte, and so do a random 256^3 region,
  the whole field at downsampling 2 2 2 and a region at a coarser tolerance.
* Tolerance 1e-5 (the decode sweep; the reference clamps the decode tolerance up to the
  encode tolerance, Core/idx2Decode.cpp:364, so the sweep needs the finer encode): the files
  equal the reference encoder's, and decodes at tolerance {1e-1, 1e-3, 1e-5} x downsampling
  {0, 1, 2} per axis equal the reference decoder's. Full-resolution requests at the two finer
  tolerances are compared on a 384^3 region to bound the run time; the others on the whole
  field. The reference decodes with --parallel (its thread pool; output identical to its
  sequential decode)."""
import hashlib
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from idx2_files import compare_dirs

SIDE = 1024


def _tmpdir(prefix):
    return tempfile.mkdtemp(prefix=prefix, dir="/dev/shm" if os.path.isdir("/dev/shm") else None)


@pytest.fixture(scope="module")
def field3(ref_app):
    import torch
    from idx2_b200.synthetic import grf_field_torch
    tmp = _tmpdir("idx2c3_")
    f = grf_field_torch(SIDE, SIDE, SIDE, seed=7, scale="unit", n_fronts=20, device=torch.device("cuda", 0))
    raw = os.path.join(tmp, f"grf-f-[{SIDE}-{SIDE}-{SIDE}]-Float32.raw")
    f.cpu().numpy().tofile(raw)
    yield tmp, f, raw
    shutil.rmtree(tmp, ignore_errors=True)


def _encode_both(idx2g, ref_app, tmp, f, raw, tol, tag):
    ours = os.path.join(tmp, "ours" + tag)
    ref = os.path.join(tmp, "ref" + tag)
    idx2g.encode(f, out_dir=ours, name="grf", field_name="f", num_levels=3, tolerance=tol)
    r = subprocess.run([ref_app, "--encode", raw, "--num_levels", "3", "--tolerance", repr(tol), "--out_dir", ref],
                       capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stdout[-300:] + r.stderr[-300:]
    return os.path.join(ours, "grf"), os.path.join(ref, "grf")


def _ref_decode(ref_app, ds_dir, tmp, down, tol, first=None, last=None):
    out_dir = tempfile.mkdtemp(dir=tmp)
    args = [ref_app, "--decode", os.path.join(ds_dir, "f.idx2"), "--downsampling", *map(str, down),
            "--tolerance", repr(tol), "--out_dir", out_dir, "--out_file", "o.raw", "--parallel"]
    if first is not None:
        args += ["--first", *map(str, first), "--last", *map(str, last)]
    r = subprocess.run(args, capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stdout[-300:] + r.stderr[-300:]
    h = hashlib.sha256()
    with open(os.path.join(out_dir, "o.raw"), "rb") as fp:
        while True:
            b = fp.read(1 << 26)
            if not b:
                break
            h.update(b)
    shutil.rmtree(out_dir, ignore_errors=True)
    return h.hexdigest()


def _our_decode(ds, down, tol, first=None, last=None):
    import torch
    _, dims, _ = ds.output_grid(first, last, down)
    out = torch.empty((dims[2], dims[1], dims[0]), dtype=torch.float32, device="cuda")
    ds.decode(first=first, last=last, downsampling=down, tolerance=tol, out=out)
    h = hashlib.sha256()
    flat = out.reshape(-1)
    step = 1 << 24
    for i in range(0, flat.numel(), step):
        h.update(flat[i:i + step].cpu().numpy().tobytes())
    return h.hexdigest()


@pytest.mark.gpu
def test_config3_tol1e3_files_and_decodes_match_reference(idx2g, ref_app, field3):
    tmp, f, raw = field3
    ours, ref = _encode_both(idx2g, ref_app, tmp, f, raw, 1e-3, "3")
    try:
        diffs = compare_dirs(ref, ours)
        assert diffs == [], diffs[:5]
        rng = np.random.default_rng(11)
        first = [int(v) for v in rng.integers(0, SIDE - 256, 3)]
        last = [v + 255 for v in first]
        ds = idx2g.Dataset(os.path.join(ours, "f.idx2"))
        for down, tol, fl in (((0, 0, 0), 0.0, None), ((0, 0, 0), 0.0, (first, last)),
                              ((2, 2, 2), 0.0, None), ((1, 0, 1), 1e-1, (first, last))):
            a, b = (fl if fl else (None, None))
            assert _our_decode(ds, down, tol, a, b) == _ref_decode(ref_app, ours, tmp, down, tol, a, b), (down, tol, fl)
        ds.close()
    finally:
        shutil.rmtree(os.path.dirname(ours), ignore_errors=True)
        shutil.rmtree(os.path.dirname(ref), ignore_errors=True)


@pytest.mark.gpu
def test_config3_tol1e5_sweep_matches_reference(idx2g, ref_app, field3):
    tmp, f, raw = field3
    ours, ref = _encode_both(idx2g, ref_app, tmp, f, raw, 1e-5, "5")
    try:
        diffs = compare_dirs(ref, ours)
        assert diffs == [], diffs[:5]
        shutil.rmtree(os.path.dirname(ref), ignore_errors=True)
        ds = idx2g.Dataset(os.path.join(ours, "f.idx2"))
        rng = np.random.default_rng(12)
        first = [int(v) for v in rng.integers(0, SIDE - 384, 3)]
        last = [v + 383 for v in first]
        for tol in (1e-1, 1e-3, 1e-5):
            for d in (0, 1, 2):
                down = (d, d, d)
                fl = (first, last) if (d == 0 and tol < 1e-1) else (None, None)
                assert _our_decode(ds, down, tol, *fl) == _ref_decode(ref_app, ours, tmp, down, tol, *fl), (down, tol)
        # mixed per-axis downsampling
        for down in ((0, 1, 2), (2, 0, 1)):
            assert _our_decode(ds, down, 1e-3) == _ref_decode(ref_app, ours, tmp, down, 1e-3), down
        ds.close()
    finally:
        shutil.rmtree(os.path.dirname(ours), ignore_errors=True)
        shutil.rmtree(os.path.dirname(ref), ignore_errors=True)


@pytest.mark.gpu
def test_config3_full_decode_error(idx2g, field3):
    """The measured error of the full-resolution decode at 1e-3 (not a parity gate: the
    reference does not bound pointwise error by the tolerance; 0.0124 measured)."""
    import torch
    tmp, f, raw = field3
    d = os.path.join(tmp, "err")
    idx2g.encode(f, out_dir=d, name="grf", field_name="f", num_levels=3, tolerance=1e-3)
    ds = idx2g.Dataset(os.path.join(d, "grf", "f.idx2"))
    out = torch.empty_like(f)
    ds.decode(out=out)
    ds.close()
    shutil.rmtree(d, ignore_errors=True)
    err = float((out - f).abs().max())
    assert err < 2e-2, err
