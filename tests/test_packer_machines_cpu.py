"""Property test of the packer's two channel state machines (the library's plan, packer and
writer driven by the oracle's CPU brick coder): over seeded random fields, dims, levels,
tolerances, types and chunk/file sizes, the machine that runs each (level, subband) over its
chunk ranges in parallel writes the same dataset files, byte for byte, as the one that runs
event by event (IDX2G_PACK_SEQUENTIAL)."""
import os
import subprocess

import numpy as np
import pytest

from idx2_files import compare_dirs
from oracle_tools import build_oracle_encode


def _cases(n, seed):
    """n parameter sets the format rules accept (drawn, checked, kept)."""
    import idx2_b200
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        is2d = rng.integers(0, 4) == 0
        dims = [int(rng.integers(33, 130)), int(rng.integers(33, 130)), 1 if is2d else int(rng.integers(33, 100))]
        c = dict(dims=dims, dtype="float32" if rng.integers(0, 2) else "float64",
                 levels=int(rng.integers(1, 3)), tol=float(10.0 ** rng.uniform(-6, -2)),
                 bpc=int(2 ** rng.integers(0, 4)), cpf=int(2 ** rng.integers(0, 3)),
                 fpd=int(2 ** rng.integers(1, 4)), seed=int(rng.integers(1 << 30)))
        p = idx2_b200.Params(dims=dims, dtype=c["dtype"], brick_dims=(32, 32, 1 if is2d else 32),
                             num_levels=c["levels"], tolerance=c["tol"], bricks_per_chunk=c["bpc"],
                             chunks_per_file=c["cpf"], files_per_dir=c["fpd"])
        if idx2_b200.check_params(p) == 0:
            out.append(c)
    return out


def _encode(exe, raw, c, out, sequential):
    nx, ny, nz = c["dims"]
    brick = [32, 32, 1 if nz == 1 else 32]
    args = [exe, raw, str(nx), str(ny), str(nz), c["dtype"], str(c["levels"]), repr(c["tol"]), out, "kat", "f"]
    args += [str(b) for b in brick] + [str(c["bpc"]), str(c["cpf"]), str(c["fpd"])]
    env = dict(os.environ)
    env.pop("IDX2G_PACK_SEQUENTIAL", None)
    if sequential:
        env["IDX2G_PACK_SEQUENTIAL"] = "1"
    return subprocess.run(args, capture_output=True, text=True, env=env)


@pytest.mark.parametrize("c", _cases(16, seed=2024), ids=lambda c: "x".join(map(str, c["dims"])) + f"-{c['dtype']}-bpc{c['bpc']}")
def test_chunk_range_machine_equals_sequential(tmp_path, c):
    from idx2_b200.synthetic import bumps_field
    exe = build_oracle_encode()
    nx, ny, nz = c["dims"]
    f = bumps_field(nx, ny, nz, seed=c["seed"]).astype(np.float32 if c["dtype"] == "float32" else np.float64)
    raw = str(tmp_path / "in.raw")
    f.tofile(raw)
    r1 = _encode(exe, raw, c, str(tmp_path / "chunk"), False)
    r2 = _encode(exe, raw, c, str(tmp_path / "seq"), True)
    assert r1.returncode == 0 and r2.returncode == 0, (r1.stderr[-300:], r2.stderr[-300:])
    assert compare_dirs(str(tmp_path / "seq" / "kat"), str(tmp_path / "chunk" / "kat")) == []
