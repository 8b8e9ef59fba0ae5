"""The file writer on the CPU (the library's plan, packer and writer driven by the oracle's
brick coder): data files of 64 MB and more are written through a mapping of the file and keep
the pages of an older file of the same name (size set first, every byte written). Encodes
into a directory that already holds a larger, a smaller or a small-file dataset of the same
name give the bytes of an encode into a fresh directory."""
import os

import numpy as np
import pytest

from idx2_files import compare_dirs
from oracle_tools import oracle_encode

DIMS = (320, 256, 256)  # float64 noise: a level-0 file of 70 to 90 MB


def _encode(tmp, f, tol, out):
    raw = os.path.join(tmp, "in.raw")
    f.tofile(raw)
    rc, err = oracle_encode(raw, DIMS, "float64", 2, tol, out, name="kat", field="f")
    os.remove(raw)
    assert rc == 0, err
    return os.path.join(out, "kat")


def _file_sizes(d):
    return sorted(os.path.getsize(os.path.join(r, n)) for r, _, fs in os.walk(d) for n in fs)


def test_reused_file_names_match_fresh_encodes(tmp_path):
    tmp = str(tmp_path)
    rng = np.random.default_rng(5)
    noise = lambda: rng.random((DIMS[2], DIMS[1], DIMS[0]))  # noqa: E731
    z, y, x = np.meshgrid(*[np.linspace(0, 1, n) for n in (DIMS[2], DIMS[1], DIMS[0])], indexing="ij")
    smooth = np.sin(3 * x) * np.cos(2 * y) + z * z
    steps = [(noise(), 1e-10), (noise(), 1e-8), (smooth, 1e-3), (noise(), 1e-10)]
    shared = os.path.join(tmp, "shared")
    for i, (f, tol) in enumerate(steps):
        fresh = _encode(tmp, f, tol, os.path.join(tmp, f"fresh{i}"))
        reused = _encode(tmp, f, tol, shared)
        assert compare_dirs(fresh, reused) == [], i
        if i != 2:
            assert max(_file_sizes(fresh)) >= 64 << 20, "the case should take the mapped write"
