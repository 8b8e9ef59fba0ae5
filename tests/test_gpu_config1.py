"""The plain CPU-runnable workload at full size: one 384x384x256 float64 field (64 Gaussian
bumps, sin/cos products at wavenumbers 1-4, N(0, 1e-4) noise; seed 1234), 2 levels, 32^3
bricks, tolerance 1e-3, decoded at downsampling 0 0 0 and 1 1 1. Dataset files against the
reference encoder's, decoded grids against the reference decoder's, byte for byte."""
import os
import subprocess

import numpy as np
import pytest

from idx2_files import compare_dirs

DIMS = (384, 384, 256)


@pytest.fixture(scope="module")
def config1(tmp_path_factory, ref_app):
    from idx2_b200.synthetic import bumps_field
    tmp = str(tmp_path_factory.mktemp("config1"))
    f = bumps_field(*DIMS, seed=1234).astype(np.float64)
    raw = os.path.join(tmp, "Miranda-Viscosity-[384-384-256]-Float64.raw")
    f.tofile(raw)
    r = subprocess.run([ref_app, "--encode", raw, "--num_levels", "2", "--tolerance", "0.001",
                        "--out_dir", os.path.join(tmp, "ref")], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-300:] + r.stderr[-300:]
    return tmp, f


@pytest.mark.gpu
def test_config1_encode_matches_reference(idx2g, config1):
    tmp, f = config1
    idx2g.encode(f, out_dir=os.path.join(tmp, "ours"), name="Miranda", field_name="Viscosity", num_levels=2,
                 tolerance=1e-3)
    diffs = compare_dirs(os.path.join(tmp, "ref", "Miranda"), os.path.join(tmp, "ours", "Miranda"))
    assert diffs == [], diffs[:5]


@pytest.mark.gpu
@pytest.mark.parametrize("down", [(0, 0, 0), (1, 1, 1)])
def test_config1_decode_matches_reference(idx2g, ref_app, config1, down):
    tmp, f = config1
    idx2_file = os.path.join(tmp, "ref", "Miranda", "Viscosity.idx2")
    out_dir = os.path.join(tmp, "refout%d" % down[0])
    os.makedirs(out_dir, exist_ok=True)
    r = subprocess.run([ref_app, "--decode", idx2_file, "--downsampling", *map(str, down), "--out_dir", out_dir,
                        "--out_file", "o.raw"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-300:] + r.stderr[-300:]
    ref = open(os.path.join(out_dir, "o.raw"), "rb").read()
    ds = idx2g.Dataset(idx2_file)
    got = ds.decode(downsampling=down)
    ds.close()
    assert got.tobytes() == ref
    if down == (0, 0, 0):
        # the reference's own error at tolerance 1e-3 (it does not bound the pointwise error)
        assert float(np.abs(got - f).max()) < 1e-2
