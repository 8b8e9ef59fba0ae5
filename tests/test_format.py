"""Host format logic (Finalize, brick/chunk/file orders, error codes) against the
reference's tables (tests/golden/kats.json), and the library's C-ABI validation."""
import json
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
KATS = json.load(open(os.path.join(HERE, "golden", "kats.json")))


@pytest.fixture(scope="module")
def format_dump():
    build = os.path.join(HERE, "_build")
    os.makedirs(build, exist_ok=True)
    exe = os.path.join(build, "format_dump")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I" + os.path.join(ROOT, "idx2_b200", "csrc"),
                    os.path.join(HERE, "cpp", "format_dump.cpp"),
                    os.path.join(ROOT, "idx2_b200", "csrc", "format.cpp"), "-o", exe], check=True)
    return exe


def test_finalize_tables_match_reference(format_dump):
    cases = KATS["finalize"]
    lines = "\n".join(" ".join(map(str, c["dims"] + [0 if c["dtype"] == "float32" else 1] + c["brick"] +
                                   [c["levels"], c["bpc"], c["cpf"], c["fpd"]])) for c in cases)
    out = subprocess.run([format_dump], input=lines + "\n", capture_output=True, text=True, check=True)
    rows = out.stdout.strip().split("\n")
    assert len(rows) == len(cases)
    n_ok = 0
    for c, row in zip(cases, rows):
        parts = row.split("|")
        head = parts[0].split()
        assert int(head[0]) == c["code"], (c, row[:80])
        if c["code"] != 0:
            continue
        n_ok += 1
        L = int(head[1])
        assert L == c["nlevels"] and list(map(int, head[2:5])) == c["group3"]
        assert list(map(int, parts[1].split())) == c["i32"], c
        assert list(map(int, parts[2].split())) == c["u64"], c
        strs = [s if s != "-" else "" for s in parts[3].split()]
        assert [strs[3 * l:3 * l + 3] for l in range(L)] == c["strs"], c
    # the uneven-field set exercises both accepted and rejected shapes
    assert 200 < n_ok < len(cases)


def test_check_params_codes_through_cabi(idx2g):
    for c in KATS["finalize"][:200]:
        p = idx2g.Params(dims=c["dims"], dtype=c["dtype"], brick_dims=c["brick"], num_levels=c["levels"],
                         tolerance=1e-3, bricks_per_chunk=c["bpc"], chunks_per_file=c["cpf"],
                         files_per_dir=c["fpd"])
        assert idx2g.check_params(p) == c["code"], c


def test_error_names(idx2g):
    assert idx2g.error_string(0) == "NoError"
    assert idx2g.error_string(22) == "BrickSizeTooBig"
    assert idx2g.error_string(23) == "TooManyLevels"
    assert idx2g.error_string(37) == "FileNotFound"


def test_brick_linearizer_equals_linear_brick():
    """The table form of the linear brick index (used by the decode plan) gives linear_brick's
    index for every brick of every level, and past the tables, over 3D and 2D shapes with
    unequal sides and partial bricks."""
    build = os.path.join(HERE, "_build")
    os.makedirs(build, exist_ok=True)
    exe = os.path.join(build, "linearizer_check")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I" + os.path.join(ROOT, "idx2_b200", "csrc"),
                    os.path.join(HERE, "cpp", "linearizer_check.cpp"),
                    os.path.join(ROOT, "idx2_b200", "csrc", "format.cpp"), "-o", exe], check=True)
    cases = ["256 256 256 32 32 32 3", "1024 512 300 32 32 32 3", "100 90 75 32 32 32 2", "300 200 1 32 32 1 2",
             "65 66 97 32 32 32 2", "513 257 129 16 16 16 4"]
    out = subprocess.run([exe], input="\n".join(cases) + "\n", capture_output=True, text=True)
    rows = out.stdout.split("\n")[:len(cases)]
    assert out.returncode == 0, out.stdout
    assert all(r.startswith("ok ") and int(r.split()[1]) > 0 for r in rows), rows
