"""Data files of 64 MB and more are written through a mapping of the file, keep the pages of a
file of the same name (its size is set first, then every byte written), and get their pages
allocated ahead (while the device stage runs) from the sizes of the previous encode of the
same shape. Encodes into fresh and into reused directories, with larger and smaller files
before them, give the reference encoder's files."""
import os
import subprocess

import numpy as np
import pytest

from idx2_files import compare_dirs

DIMS = (320, 256, 256)  # x, y, z; float64 noise: data files of 70 to 90 MB


def _noise(seed):
    rng = np.random.default_rng(seed)
    return rng.random((DIMS[2], DIMS[1], DIMS[0]))


def _smooth(seed):
    from idx2_b200.synthetic import bumps_field
    return bumps_field(DIMS[0], DIMS[1], DIMS[2], seed=seed).astype(np.float64)


def _ref(ref_app, tmp, f, tol, tag):
    raw = os.path.join(tmp, f"kat-f-[{DIMS[0]}-{DIMS[1]}-{DIMS[2]}]-Float64.raw")
    f.tofile(raw)
    out = os.path.join(tmp, "ref_" + tag)
    r = subprocess.run([ref_app, "--encode", raw, "--num_levels", "2", "--tolerance", repr(tol), "--out_dir", out],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-300:] + r.stderr[-300:]
    os.remove(raw)
    return os.path.join(out, "kat")


@pytest.mark.gpu
def test_reused_and_preallocated_files_match_reference(idx2g, ref_app, tmp_path):
    tmp = str(tmp_path)
    steps = [
        # field, tolerance, directory, reference tag
        (_noise(1), 1e-10, "a", "n1"),
        (_noise(2), 1e-10, "b", "n2"),     # fresh directory, pages allocated ahead
        (_noise(2), 1e-10, "a", "n2"),     # same names as a larger-or-equal older file
        (_noise(3), 1e-8, "a", "n3"),      # a smaller large file over a larger one
        (_smooth(4), 1e-3, "a", "s4"),     # small files (truncated) over large ones
        (_noise(5), 1e-10, "a", "n5"),     # large files over small ones
    ]
    refs = {}
    for f, tol, d, tag in steps:
        if tag not in refs:
            refs[tag] = _ref(ref_app, tmp, f, tol, tag)
        # one dataset name throughout: later encodes into a directory reuse its file names
        out = os.path.join(tmp, d)
        info = idx2g.encode(f, out_dir=out, name="kat", field_name="f", num_levels=2, tolerance=tol)
        diffs = compare_dirs(refs[tag], os.path.join(out, "kat"))
        assert diffs == [], (d, tag, diffs[:3])
        if tag.startswith("n"):
            assert info.file_bytes > 64 << 20
