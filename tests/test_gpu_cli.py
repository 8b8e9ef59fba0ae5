"""The idx2App-compatible CLI (idx2_b200/idx2g_app) against the reference CLI (oracle/_ref
idx2App), run the way a user runs them: --encode of a raw file (name, field, dims and type
from the file name; --num_levels, --tolerance, --brick_size, --out_dir) writes the same
dataset files, and --decode with --downsampling, --tolerance, --first/--last, --parallel and
--dry writes the same output file under the same default name."""
import os
import subprocess

import numpy as np
import pytest

from idx2_files import compare_dirs

HERE = os.path.dirname(os.path.abspath(__file__))
APP = os.path.join(os.path.dirname(HERE), "idx2_b200", "idx2g_app")

DECODES = [
    [],
    ["--downsampling", "1", "1", "1"],
    ["--downsampling", "2", "0", "1", "--tolerance", "0.01"],
    ["--first", "10", "5", "3", "--last", "90", "70", "60"],
    ["--first", "0", "0", "0", "--last", "63", "63", "63", "--downsampling", "1", "0", "0", "--parallel"],
    ["--tolerance", "0.1", "--parallel"],
]


def _run(args, cwd):
    r = subprocess.run(args, capture_output=True, text=True, cwd=cwd, timeout=600)
    assert r.returncode == 0, (args, r.stdout[-500:], r.stderr[-500:])
    return r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("dtype,levels,tol", [("float32", 2, 1e-3), ("float64", 2, 1e-5)])
def test_cli_encode_decode_matches_reference(ref_app, tmp_path, dtype, levels, tol):
    from idx2_b200.synthetic import bumps_field
    nx, ny, nz = 112, 96, 80
    f = bumps_field(nx, ny, nz, seed=21).astype(np.float32 if dtype == "float32" else np.float64)
    raw = tmp_path / f"cli-rho-[{nx}-{ny}-{nz}]-{dtype.capitalize()}.raw"
    f.tofile(raw)
    for app, sub in ((ref_app, "ref"), (APP, "ours")):
        _run([app, "--encode", str(raw), "--num_levels", str(levels), "--tolerance", str(tol),
              "--out_dir", str(tmp_path / sub)], str(tmp_path))
    assert compare_dirs(str(tmp_path / "ref" / "cli"), str(tmp_path / "ours" / "cli")) == []
    for k, extra in enumerate(DECODES):
        outs = []
        for app, sub in ((ref_app, "ref"), (APP, "ours")):
            od = tmp_path / f"out_{sub}_{k}"
            od.mkdir()
            _run([app, "--decode", str(tmp_path / sub / "cli" / "rho.idx2"), "--out_dir", str(od)] + extra,
                 str(tmp_path))
            files = sorted(os.listdir(od))
            assert len(files) == 1, files
            outs.append((files[0], (od / files[0]).read_bytes()))
        # the default output name (Core/idx2Decode.cpp:344-345) and the bytes
        assert outs[0][0] == outs[1][0], (extra, outs[0][0], outs[1][0])
        assert outs[0][1] == outs[1][1], extra
    # --dry decodes and writes nothing
    od = tmp_path / "dry"
    od.mkdir()
    _run([APP, "--decode", str(tmp_path / "ours" / "cli" / "rho.idx2"), "--out_dir", str(od), "--dry"], str(tmp_path))
    assert os.listdir(od) == []
