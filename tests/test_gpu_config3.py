"""The headline workload at full size: a 1024^3 float32 k^-5/3 Gaussian random field (seeded,
unit variance) with 20 tanh fronts, 3 levels, 32^3 bricks, tolerance 1e-3, encoded by this
library. The reference decoder reads the same files: a random 256^3 region at full
resolution, the whole field at downsampling 2 2 2, and a region at a coarser tolerance decode
byte for byte like this library's decoder (the reference CPU encode of 4.3 GB is too slow for a
test; the encoder's file parity is covered at smaller sizes). The full-resolution decode stays
within the reference decoder's error behaviour at this tolerance."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

SIDE = 1024


@pytest.fixture(scope="module")
def config3(ref_app):
    import torch
    import idx2_b200
    from idx2_b200.synthetic import grf_field_torch
    tmp = tempfile.mkdtemp(prefix="idx2c3_", dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
    f = grf_field_torch(SIDE, SIDE, SIDE, seed=7, scale="unit", n_fronts=20, device=torch.device("cuda", 0))
    idx2_b200.encode(f, out_dir=tmp, name="grf", field_name="f", num_levels=3, tolerance=1e-3)
    yield tmp, f
    shutil.rmtree(tmp, ignore_errors=True)


def _ref(ref_app, tmp, tag, down, tol, first=None, last=None):
    out_dir = os.path.join(tmp, "refout_" + tag)
    os.makedirs(out_dir, exist_ok=True)
    args = [ref_app, "--decode", os.path.join(tmp, "grf", "f.idx2"), "--downsampling", *map(str, down),
            "--tolerance", repr(tol), "--out_dir", out_dir, "--out_file", "o.raw"]
    if first is not None:
        args += ["--first", *map(str, first), "--last", *map(str, last)]
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-300:] + r.stderr[-300:]
    data = open(os.path.join(out_dir, "o.raw"), "rb").read()
    shutil.rmtree(out_dir, ignore_errors=True)
    return data


@pytest.mark.gpu
@pytest.mark.parametrize("req", ["roi", "ds2", "roi_coarse"])
def test_config3_decode_matches_reference(idx2g, ref_app, config3, req):
    tmp, f = config3
    rng = np.random.default_rng(11)
    first = [int(v) for v in rng.integers(0, SIDE - 256, 3)]
    last = [v + 255 for v in first]
    ds = idx2g.Dataset(os.path.join(tmp, "grf", "f.idx2"))
    if req == "roi":
        got = ds.decode(first=first, last=last)
        ref = _ref(ref_app, tmp, req, (0, 0, 0), 0.0, first, last)
    elif req == "ds2":
        got = ds.decode(downsampling=(2, 2, 2))
        ref = _ref(ref_app, tmp, req, (2, 2, 2), 0.0)
    else:
        got = ds.decode(first=first, last=last, downsampling=(1, 0, 1), tolerance=1e-1)
        ref = _ref(ref_app, tmp, req, (1, 0, 1), 1e-1, first, last)
    ds.close()
    assert got.tobytes() == ref


@pytest.mark.gpu
def test_config3_full_decode_error(idx2g, config3):
    import torch
    tmp, f = config3
    ds = idx2g.Dataset(os.path.join(tmp, "grf", "f.idx2"))
    out = torch.empty_like(f)
    ds.decode(out=out)
    ds.close()
    # the reference decoder does not bound the pointwise error by the tolerance; on this
    # workload the decode error stays near 1e-2 (0.0124 measured)
    err = float((out - f).abs().max())
    assert err < 2e-2, err
