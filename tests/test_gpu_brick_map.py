"""Brick-map decode (the reference's HashMap output, idx2App --brick_map) against the reference
CLI's `bricks` file, byte for byte: the significant-brick selection, the per-brick resolution
and the FP64 samples of every record."""
import os
import struct
import subprocess

import numpy as np
import pytest


IDX2G_APP = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "idx2_b200", "idx2g_app")


def _flat_slab_field(nx, ny, nz, seed):
    """Bumps with flat slabs inside the coarsest bricks: their finest bricks carry no detail,
    so the map mixes full-resolution records with records from the coarser level (every
    coarsest brick keeps detail elsewhere: the reference fails on a chain with no significant
    brick)."""
    from idx2_b200.synthetic import bumps_field
    f = bumps_field(nx, ny, nz, seed=seed)
    f[:, :, 32:64] = 0.0
    f[:32, 64:128, 96:128] = 0.25
    return f


def _encode_ref_field(ref_app, tmp, f, name, levels, tol, bd):
    nz, ny, nx = f.shape
    dt = "Float32" if f.dtype == np.float32 else "Float64"
    raw = os.path.join(tmp, f"kat-{name}-[{nx}-{ny}-{nz}]-{dt}.raw")
    f.tofile(raw)
    args = [ref_app, "--encode", raw, "--num_levels", str(levels), "--tolerance", str(tol),
            "--out_dir", os.path.join(tmp, "ds")]
    if bd[2] == 1:
        args += ["--brick_size", "32", "32", "1"]
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-300:]
    return os.path.join(tmp, "ds", "kat", f"{name}.idx2")


def _ref_bricks(ref_app, tmp, idx2_file, opts):
    d = os.path.join(tmp, "ref_" + "_".join(o.replace(".", "p") for o in opts))
    os.makedirs(d, exist_ok=True)
    r = subprocess.run([ref_app, "--decode", idx2_file, "--brick_map", *opts, "--out_dir", d],
                       capture_output=True, text=True, cwd=d)
    assert r.returncode == 0, r.stdout[-300:] + r.stderr[-300:]
    return open(os.path.join(d, "bricks"), "rb").read()


def _records(b):
    """(brick, dims) of every record of a bricks file."""
    out, off = [], 36
    while off < len(b):
        b3 = struct.unpack("3i", b[off:off + 12])
        d3 = struct.unpack("3i", b[off + 12:off + 24])
        off += 24 + 8 * d3[0] * d3[1] * d3[2]
        out.append((b3, d3))
    return out


CASES = [
    # field, levels, encode tol, brick dims, decode options
    ("slab", 2, 1e-3, (32, 32, 32), []),
    ("slab", 2, 1e-3, (32, 32, 32), ["--downsampling", "1", "1", "1"]),
    ("slab", 2, 1e-3, (32, 32, 32), ["--tolerance", "0.1"]),
    ("bumps64", 2, 1e-3, (32, 32, 32), []),
    ("plane", 2, 1e-3, (32, 32, 1), []),
]


def _field(kind):
    from idx2_b200.synthetic import bumps_field
    if kind == "slab":
        return _flat_slab_field(160, 160, 96, 5).astype(np.float32)
    if kind == "bumps64":
        return bumps_field(96, 80, 72, seed=3).astype(np.float64)
    return bumps_field(200, 150, 1, seed=7).astype(np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("ci", range(len(CASES)))
def test_brick_map_matches_reference(idx2g, ref_app, tmp_path, ci):
    kind, levels, tol, bd, opts = CASES[ci]
    tmp = str(tmp_path)
    idx2_file = _encode_ref_field(ref_app, tmp, _field(kind), "g", levels, tol, bd)
    ref = _ref_bricks(ref_app, tmp, idx2_file, opts)
    ds_ = (0, 0, 0)
    dtol = 0.0
    if "--downsampling" in opts:
        i = opts.index("--downsampling")
        ds_ = tuple(int(x) for x in opts[i + 1:i + 4])
    if "--tolerance" in opts:
        dtol = float(opts[opts.index("--tolerance") + 1])
    ds = idx2g.Dataset(idx2_file)
    ours = os.path.join(tmp, "ours_bricks")
    ds.decode_brick_map(ours, downsampling=ds_, tolerance=dtol)
    ds.close()
    got = open(ours, "rb").read()
    assert got[:36] == ref[:36]
    assert _records(got) == _records(ref)
    assert got == ref
    if kind == "slab" and not opts:
        # the map mixes full-resolution and coarser records
        assert {d for _, d in _records(got)} == {(33, 33, 33), (17, 17, 17)}


@pytest.mark.gpu
def test_brick_map_cli(idx2g, ref_app, tmp_path):
    """idx2g_app --decode ... --brick_map writes the same `bricks` file as idx2App."""
    if not os.path.exists(IDX2G_APP):
        pytest.skip("idx2g_app not built")
    tmp = str(tmp_path)
    idx2_file = _encode_ref_field(ref_app, tmp, _field("slab"), "g", 2, 1e-3, (32, 32, 32))
    ref = _ref_bricks(ref_app, tmp, idx2_file, [])
    d = os.path.join(tmp, "cli")
    os.makedirs(d)
    r = subprocess.run([IDX2G_APP, "--decode", idx2_file, "--brick_map"], capture_output=True, text=True, cwd=d)
    assert r.returncode == 0, r.stdout[-300:] + r.stderr[-300:]
    assert open(os.path.join(d, "bricks"), "rb").read() == ref


@pytest.mark.gpu
def test_brick_map_of_own_encode(idx2g, ref_app, tmp_path):
    """A dataset written by this library maps to the same bricks file with either decoder."""
    tmp = str(tmp_path)
    f = _field("slab")
    idx2g.encode(f, out_dir=os.path.join(tmp, "ds"), name="kat", field_name="g", num_levels=2, tolerance=1e-3)
    idx2_file = os.path.join(tmp, "ds", "kat", "g.idx2")
    ref = _ref_bricks(ref_app, tmp, idx2_file, [])
    ds = idx2g.Dataset(idx2_file)
    ours = os.path.join(tmp, "ours_bricks")
    ds.decode_brick_map(ours)
    ds.close()
    assert open(ours, "rb").read() == ref
