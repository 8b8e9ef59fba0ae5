"""GPU encode parity: the CUDA library's dataset files against the reference's.

Every file must be byte-identical to the reference's, the zstd frames of the exponent
chunks and address tables included (the library writes the frames of the reference's
vendored zstd 1.4.5)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from idx2_files import compare_dirs

CASES = [
    # dims, dtype, levels, tol, brick dims, generator seed
    ((96, 80, 72), "float64", 2, 1e-3, (32, 32, 32), 3),
    ((64, 64, 64), "float32", 1, 1e-3, (32, 32, 32), 4),
    ((130, 70, 40), "float32", 1, 1e-4, (32, 32, 32), 5),
    ((128, 128, 128), "float64", 2, 1e-5, (32, 32, 32), 6),
    ((200, 150, 1), "float32", 2, 1e-3, (32, 32, 1), 7),
    ((160, 128, 96), "float32", 2, 1e-3, (32, 32, 32), 8),
    ((33, 47, 65), "float64", 1, 1e-6, (32, 32, 32), 9),
]


def _field(dims, dtype, seed):
    from idx2_b200.synthetic import bumps_field
    nx, ny, nz = dims
    return bumps_field(nx, ny, nz, seed=seed).astype(np.float32 if dtype == "float32" else np.float64)


def _ref_encode(ref_app, tmp, f, dims, dtype, levels, tol, bd):
    nx, ny, nz = dims
    raw = os.path.join(tmp, f"kat-f-[{nx}-{ny}-{nz}]-{dtype.capitalize()}.raw")
    f.tofile(raw)
    args = [ref_app, "--encode", raw, "--num_levels", str(levels), "--tolerance", str(tol),
            "--out_dir", os.path.join(tmp, "ref")]
    if bd[2] == 1:
        args += ["--brick_size", "32", "32", "1"]
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-500:] + r.stderr[-500:]
    return os.path.join(tmp, "ref", "kat")


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}-{c[1]}-L{c[2]}-{c[3]}" for c in CASES])
def test_encode_matches_reference(idx2g, ref_app, tmp_path, case):
    dims, dtype, levels, tol, bd, seed = case
    f = _field(dims, dtype, seed)
    ref_dir = _ref_encode(ref_app, str(tmp_path), f, dims, dtype, levels, tol, bd)
    info = idx2g.encode(f, out_dir=str(tmp_path / "ours"), name="kat", field_name="f",
                        num_levels=levels, tolerance=tol, brick_dims=bd)
    assert info.kernel_launches >= levels
    diffs = compare_dirs(ref_dir, str(tmp_path / "ours" / "kat"))
    assert diffs == [], diffs[:5]


@pytest.mark.gpu
def test_encode_from_device_tensor(idx2g, ref_app, tmp_path):
    import torch
    dims, dtype, levels, tol, bd, seed = CASES[0]
    f = _field(dims, dtype, seed)
    ref_dir = _ref_encode(ref_app, str(tmp_path), f, dims, dtype, levels, tol, bd)
    t = torch.from_numpy(f).cuda()
    idx2g.encode(t, out_dir=str(tmp_path / "ours"), name="kat", field_name="f",
                 num_levels=levels, tolerance=tol)
    assert compare_dirs(ref_dir, str(tmp_path / "ours" / "kat")) == []


def _golden_cases():
    import json
    here = os.path.dirname(os.path.abspath(__file__))
    return json.load(open(os.path.join(here, "golden", "datasets.json")))


@pytest.mark.gpu
@pytest.mark.parametrize("case", _golden_cases(), ids=lambda c: c["name"])
def test_encode_matches_golden_files(idx2g, tmp_path, case):
    """Against the committed reference output (no reference build needed)."""
    import hashlib
    from golden.golden_inputs import make_dataset_field
    f = make_dataset_field(case)
    assert hashlib.sha256(f.tobytes()).hexdigest() == case["field_sha"]
    idx2g.encode(f, out_dir=str(tmp_path), name=case["name"], field_name="f", num_levels=case["levels"],
                 tolerance=case["tol"], brick_dims=tuple(case["brick"]))
    here = os.path.dirname(os.path.abspath(__file__))
    diffs = compare_dirs(os.path.join(here, "golden", "datasets", case["name"]), str(tmp_path / case["name"]))
    assert diffs == [], diffs[:3]


@pytest.mark.gpu
@pytest.mark.parametrize("case", __import__("test_packer_chunks").CHUNK_CASES,
                         ids=__import__("test_packer_chunks").chunk_case_id)
def test_encode_chunk_boundaries_match_reference(idx2g, ref_app, tmp_path, case):
    from test_packer_chunks import chunk_field, ref_encode_chunked
    dims, dtype, levels, tol, bd, bpc, cpf, fpd, seed = case
    f = chunk_field(dims, dtype, seed)
    _, ref_dir = ref_encode_chunked(ref_app, str(tmp_path), f, case)
    idx2g.encode(f, out_dir=str(tmp_path / "ours"), name="kat", field_name="f", num_levels=levels,
                 tolerance=tol, brick_dims=bd, bricks_per_chunk=bpc, chunks_per_file=cpf,
                 files_per_dir=fpd)
    diffs = compare_dirs(ref_dir, str(tmp_path / "ours" / "kat"))
    assert diffs == [], diffs[:5]
