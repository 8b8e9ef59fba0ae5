"""The library's host encode plan + chunk packer, driven by the oracle's CPU brick
coder, against the reference's dataset files (tests/golden/datasets)."""
import json
import os
import hashlib

import pytest

from golden.golden_inputs import make_dataset_field
from idx2_files import compare_dirs
from oracle_tools import oracle_encode

HERE = os.path.dirname(os.path.abspath(__file__))
MANIFEST = json.load(open(os.path.join(HERE, "golden", "datasets.json")))


@pytest.mark.parametrize("case", MANIFEST, ids=[c["name"] for c in MANIFEST])
def test_packer_matches_reference_files(tmp_path, case):
    f = make_dataset_field(case)
    assert hashlib.sha256(f.tobytes()).hexdigest() == case["field_sha"], "input generator changed"
    raw = str(tmp_path / "in.raw")
    f.tofile(raw)
    rc, err = oracle_encode(raw, case["dims"], case["dtype"], case["levels"], case["tol"], str(tmp_path / "o"),
                            name=case["name"], field="f", brick=case["brick"])
    assert rc == 0, err
    diffs = compare_dirs(os.path.join(HERE, "golden", "datasets", case["name"]), str(tmp_path / "o" / case["name"]))
    assert diffs == [], diffs[:3]
