"""GPU decode parity: the CUDA library's decoded grids against the reference
decoder's output on the same dataset, byte for byte (FP64 inverse transform in the
reference's order, then the reference's f64 -> output dtype cast)."""
import os
import subprocess

import numpy as np
import pytest

DATASETS = [
    # dims, dtype, levels, encode tol, brick dims, seed
    ((96, 80, 72), "float64", 2, 1e-3, (32, 32, 32), 3),
    ((160, 128, 96), "float32", 2, 1e-3, (32, 32, 32), 8),
    ((256, 256, 256), "float32", 3, 1e-5, (32, 32, 32), 12),
    ((200, 150, 1), "float32", 2, 1e-3, (32, 32, 1), 7),
    ((130, 70, 40), "float64", 1, 1e-4, (32, 32, 32), 5),
]

REQUESTS = [
    # downsampling, decode tolerance, (first, last) or None
    ((0, 0, 0), 0.0, None),
    ((1, 1, 1), 0.0, None),
    ((2, 2, 2), 0.0, None),
    ((0, 1, 2), 0.0, None),
    ((0, 0, 0), 1e-1, None),
    ((0, 0, 0), 0.0, "roi"),
    ((1, 0, 1), 1e-2, "roi"),
]


def _encode_ref(ref_app, tmp, dims, dtype, levels, tol, bd, seed):
    from idx2_b200.synthetic import bumps_field
    nx, ny, nz = dims
    f = bumps_field(nx, ny, nz, seed=seed).astype(np.float32 if dtype == "float32" else np.float64)
    raw = os.path.join(tmp, f"kat-f-[{nx}-{ny}-{nz}]-{dtype.capitalize()}.raw")
    f.tofile(raw)
    args = [ref_app, "--encode", raw, "--num_levels", str(levels), "--tolerance", str(tol),
            "--out_dir", os.path.join(tmp, "ds")]
    if bd[2] == 1:
        args += ["--brick_size", "32", "32", "1"]
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-300:]
    return f, os.path.join(tmp, "ds", "kat", "f.idx2")


def _roi(dims):
    first = [d // 5 for d in dims]
    last = [max(f, (3 * d) // 4) for f, d in zip(first, dims)]
    return first, last


def _ref_decode(ref_app, tmp, idx2_file, ds, tol, roi, dims):
    out_dir = os.path.join(tmp, "refout")
    os.makedirs(out_dir, exist_ok=True)
    args = [ref_app, "--decode", idx2_file, "--downsampling", *map(str, ds), "--tolerance", repr(tol),
            "--out_dir", out_dir, "--out_file", "o.raw"]
    if roi:
        first, last = _roi(dims)
        args += ["--first", *map(str, first), "--last", *map(str, last)]
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-300:] + r.stderr[-300:]
    return open(os.path.join(out_dir, "o.raw"), "rb").read()


@pytest.mark.gpu
@pytest.mark.parametrize("dsi", range(len(DATASETS)))
def test_decode_matches_reference(idx2g, ref_app, tmp_path, dsi):
    dims, dtype, levels, tol, bd, seed = DATASETS[dsi]
    tmp = str(tmp_path)
    _, idx2_file = _encode_ref(ref_app, tmp, dims, dtype, levels, tol, bd, seed)
    ds = idx2g.Dataset(idx2_file)
    for down, dtol, roi in REQUESTS:
        if bd[2] == 1:
            down = (down[0], down[1], 0)
        if max(down) >= levels + 1:
            continue
        first = last = None
        if roi:
            first, last = _roi(dims)
        ours = ds.decode(first=first, last=last, downsampling=down, tolerance=dtol)
        ref = _ref_decode(ref_app, tmp, idx2_file, down, dtol, roi, dims)
        assert ours.tobytes() == ref, (down, dtol, roi, ours.shape)
    ds.close()


@pytest.mark.gpu
def test_roundtrip_own_files(idx2g, ref_app, tmp_path):
    """Our encoder's files decode identically with the reference decoder and ours."""
    from idx2_b200.synthetic import bumps_field
    f = bumps_field(128, 96, 80, seed=21).astype(np.float32)
    idx2g.encode(f, out_dir=str(tmp_path / "o"), name="kat", field_name="f", num_levels=2, tolerance=1e-3)
    idx2_file = str(tmp_path / "o" / "kat" / "f.idx2")
    ds = idx2g.Dataset(idx2_file)
    ours = ds.decode()
    ref = _ref_decode(ref_app, str(tmp_path), idx2_file, (0, 0, 0), 0.0, None, (128, 96, 80))
    assert ours.tobytes() == ref
    err = np.abs(ours.astype(np.float64) - f.astype(np.float64)).max()
    assert err < 1e-2, err


def _golden_cases():
    import json
    here = os.path.dirname(os.path.abspath(__file__))
    return json.load(open(os.path.join(here, "golden", "datasets.json")))


@pytest.mark.gpu
@pytest.mark.parametrize("case", _golden_cases(), ids=lambda c: c["name"])
def test_decode_matches_golden(idx2g, tmp_path, case):
    """Decode the committed reference datasets; compare with the reference decoder's output
    digests (no reference build needed)."""
    import hashlib
    import shutil
    here = os.path.dirname(os.path.abspath(__file__))
    src = os.path.join(here, "golden", "datasets")
    shutil.copytree(src, str(tmp_path / "ds"))
    ds = idx2g.Dataset(str(tmp_path / "ds" / case["name"] / "f.idx2"))
    for req in case["decodes"]:
        out = ds.decode(first=req.get("first"), last=req.get("last"), downsampling=req["ds"], tolerance=req["tol"])
        assert out.nbytes == req["nbytes"], req
        assert hashlib.sha256(out.tobytes()).hexdigest() == req["sha"], req
    ds.close()
