"""Chunk, file and directory boundaries: the library's host plan + packer, driven by the
oracle's CPU brick coder, against the reference CLI (oracle/_ref/idx2App) with small
--bricks_per_chunk / --chunks_per_file / --files_per_dir, so that channels change chunk
inside a level, chunks spread over several files and files over several directories."""
import os
import subprocess

import numpy as np
import pytest

from idx2_files import compare_dirs
from oracle_tools import build_oracle_encode

# dims, dtype, levels, tol, brick dims, bricks per chunk, chunks per file, files per dir, seed
CHUNK_CASES = [
    ((160, 128, 96), "float32", 2, 1e-3, (32, 32, 32), 4, 2, 4, 11),
    ((128, 128, 128), "float64", 2, 1e-4, (32, 32, 32), 2, 4, 2, 12),
    ((256, 192, 1), "float32", 2, 1e-3, (32, 32, 1), 8, 2, 4, 13),
    ((96, 96, 96), "float32", 1, 1e-3, (32, 32, 32), 1, 1, 8, 14),
]


def chunk_case_id(c):
    return f"{c[0][0]}x{c[0][1]}x{c[0][2]}-{c[1]}-L{c[2]}-bpc{c[5]}-cpf{c[6]}-fpd{c[7]}"


def chunk_field(dims, dtype, seed):
    from idx2_b200.synthetic import bumps_field
    nx, ny, nz = dims
    return bumps_field(nx, ny, nz, seed=seed).astype(np.float32 if dtype == "float32" else np.float64)


def ref_encode_chunked(ref_app, tmp, f, case):
    dims, dtype, levels, tol, bd, bpc, cpf, fpd, _ = case
    nx, ny, nz = dims
    raw = os.path.join(tmp, f"kat-f-[{nx}-{ny}-{nz}]-{dtype.capitalize()}.raw")
    f.tofile(raw)
    args = [ref_app, "--encode", raw, "--num_levels", str(levels), "--tolerance", str(tol),
            "--out_dir", os.path.join(tmp, "ref"), "--bricks_per_chunk", str(bpc),
            "--chunks_per_file", str(cpf), "--files_per_dir", str(fpd)]
    if bd[2] == 1:
        args += ["--brick_size", "32", "32", "1"]
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-500:] + r.stderr[-500:]
    return raw, os.path.join(tmp, "ref", "kat")


@pytest.mark.parametrize("machine", ["by_chunk", "sequential"])
@pytest.mark.parametrize("case", CHUNK_CASES, ids=chunk_case_id)
def test_packer_chunk_boundaries(ref_app, tmp_path, case, machine):
    """The channel state machine run over each group's chunk ranges in parallel (the default)
    and event by event (IDX2G_PACK_SEQUENTIAL) both give the reference's files; with IDX2G_TRACE
    the packer reports how many groups took the chunk-range path (all of them here)."""
    dims, dtype, levels, tol, bd, bpc, cpf, fpd, seed = case
    f = chunk_field(dims, dtype, seed)
    raw, ref_dir = ref_encode_chunked(ref_app, str(tmp_path), f, case)
    nfiles = sum(len(fs) for _, _, fs in os.walk(ref_dir))
    assert nfiles > 3, "the case should produce several data files"
    exe = build_oracle_encode()
    args = [exe, raw, str(dims[0]), str(dims[1]), str(dims[2]), dtype, str(levels), repr(tol),
            str(tmp_path / "o"), "kat", "f"] + [str(b) for b in bd] + [str(bpc), str(cpf), str(fpd)]
    env = dict(os.environ, IDX2G_TRACE="1")
    env.pop("IDX2G_PACK_SEQUENTIAL", None)
    if machine == "sequential":
        env["IDX2G_PACK_SEQUENTIAL"] = "1"
    r = subprocess.run(args, capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stderr
    by_chunk = [ln.split() for ln in r.stderr.splitlines() if ln.startswith("idx2g pack.groups_by_chunk")]
    assert len(by_chunk) == 1
    merged, total = int(by_chunk[0][2]), int(by_chunk[0][4])
    assert merged == (total if machine == "by_chunk" else 0), by_chunk
    diffs = compare_dirs(ref_dir, str(tmp_path / "o" / "kat"))
    assert diffs == [], diffs[:3]
