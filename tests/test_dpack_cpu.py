"""The device packer's host stages (idx2_b200/csrc/dpack_plan.cpp) with its two kernels
restated on the host (tests/cpp/dpack_emul.h), driven by the oracle's CPU brick coder: the
files equal the reference's (golden datasets) and the host packer's, byte for byte, over
chunk and file boundaries (small BricksPerChunk / ChunksPerFile: many chunks per channel,
flushes in the middle of the encode, several files per level)."""
import json
import os

import numpy as np
import pytest

from golden.golden_inputs import make_dataset_field
from idx2_files import compare_dirs
from oracle_tools import oracle_encode

HERE = os.path.dirname(os.path.abspath(__file__))
MANIFEST = json.load(open(os.path.join(HERE, "golden", "datasets.json")))


@pytest.mark.parametrize("case", MANIFEST, ids=[c["name"] for c in MANIFEST])
def test_device_packer_matches_reference_files(tmp_path, case):
    f = make_dataset_field(case)
    raw = str(tmp_path / "in.raw")
    f.tofile(raw)
    rc, err = oracle_encode(raw, case["dims"], case["dtype"], case["levels"], case["tol"], str(tmp_path / "o"),
                            name=case["name"], field="f", brick=case["brick"], dpack=True)
    assert rc == 0, err
    diffs = compare_dirs(os.path.join(HERE, "golden", "datasets", case["name"]), str(tmp_path / "o" / case["name"]))
    assert diffs == [], diffs[:3]


CHUNKED = [
    # dims, dtype, levels, tol, brick, (bricks_per_chunk, chunks_per_file, files_per_dir)
    ((96, 80, 72), "float32", 2, 1e-3, (16, 16, 16), (2, 2, 64)),
    ((100, 70, 1), "float64", 3, 1e-4, (16, 16, 1), (4, 1, 64)),
    ((64, 64, 64), "float64", 1, 1e-6, (8, 8, 8), (8, 4, 64)),
    ((130, 33, 40), "float32", 2, 1e-2, (32, 16, 8), (1, 8, 64)),
]


@pytest.mark.parametrize("case", CHUNKED, ids=lambda c: f"{c[0]}-{c[1]}-L{c[2]}-b{c[4][0]}-c{c[5][0]}")
def test_device_packer_matches_host_packer_over_chunks(tmp_path, case):
    dims, dt, levels, tol, brick, chunks = case
    rng = np.random.default_rng(sum(dims) + levels)
    x, y, z = np.meshgrid(*[np.linspace(0, 1, n) for n in dims], indexing="ij")
    f = (np.sin(7 * x + 3 * y * y) * np.cos(5 * z) + 0.05 * rng.standard_normal(x.shape)).T
    f = np.ascontiguousarray(f.astype(np.float32 if dt == "float32" else np.float64))
    raw = str(tmp_path / "in.raw")
    f.tofile(raw)
    outs = {}
    for mode in ("host", "dpack"):
        rc, err = oracle_encode(raw, dims, dt, levels, tol, str(tmp_path / mode), name="c", field="f", brick=brick,
                                chunks=chunks, dpack=mode == "dpack")
        assert rc == 0, (mode, err)
        outs[mode] = str(tmp_path / mode / "c")
    nfiles = sum(len(fs) for _, _, fs in os.walk(outs["host"]))
    assert nfiles >= 3, nfiles  # several data files: chunks cross file boundaries
    assert compare_dirs(outs["host"], outs["dpack"]) == []
