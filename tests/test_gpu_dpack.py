"""The encode's packing runs on the device (dpack.cu) and equals the host packer's.

In child processes (the packer choice is read once per process): an encode traced with
IDX2G_TRACE shows the device packer's stages, and its files equal those of the same encode
with IDX2G_HOST_PACK=1 (the host packer) -- over many chunks per channel (small
BricksPerChunk, several files per level) and with several bit planes per chunk key. The
reference-parity encode tests run through the device packer as well.

Repeated encodes of one shape in one process allocate the pages of their large data files
ahead (the sizes of the previous encode, while the device works): the files they write equal
those of a fresh process, for the same field into a new directory and over the old files, and
for fields whose files come out larger or smaller than the guess."""
import os
import subprocess
import sys

import pytest

from idx2_files import compare_dirs

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

_CHILD = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
import idx2_b200
from idx2_b200.synthetic import bumps_field
dims = tuple(int(v) for v in sys.argv[3].split(","))
dt = np.float32 if sys.argv[4] == "float32" else np.float64
f = bumps_field(*dims, seed=int(sys.argv[5])).astype(dt)
idx2_b200.encode(f, out_dir=sys.argv[2], name="dp", field_name="f", num_levels=int(sys.argv[6]), tolerance=float(sys.argv[7]),
                 brick_dims=(32, 32, 1) if dims[2] == 1 else (32, 32, 32), bricks_per_chunk=int(sys.argv[8]),
                 chunks_per_file=int(sys.argv[9]), bit_planes_per_chunk=int(sys.argv[10]))
"""

CASES = [
    # dims, dtype, levels, tol, bricks_per_chunk, chunks_per_file, bit_planes_per_chunk, seed
    ((256, 192, 160), "float32", 3, 1e-3, 8, 4, 1, 61),
    ((300, 200, 1), "float64", 2, 1e-5, 4, 2, 1, 62),
    ((160, 128, 96), "float32", 2, 1e-4, 16, 64, 2, 63),
]


def _encode(out_dir, case, host_pack):
    dims, dt, levels, tol, bpc, cpf, bppc, seed = case
    env = dict(os.environ, IDX2G_TRACE="1", IDX2G_HOST_PACK="1" if host_pack else "0")
    r = subprocess.run([sys.executable, "-c", _CHILD, ROOT, out_dir, ",".join(map(str, dims)), dt, str(seed),
                        str(levels), repr(tol), str(bpc), str(cpf), str(bppc)],
                       capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stdout[-1000:] + r.stderr[-2000:]
    return r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{c[1]}-bpc{c[4]}-bp{c[6]}")
def test_device_packer_files_equal_host_packer(tmp_path, case):
    dev_log = _encode(str(tmp_path / "device"), case, host_pack=False)
    host_log = _encode(str(tmp_path / "host"), case, host_pack=True)
    assert "dpack.write" in dev_log, dev_log[-2000:]
    assert "dpack." not in host_log and "pack.channels" in host_log, host_log[-2000:]
    nfiles = sum(len(fs) for _, _, fs in os.walk(str(tmp_path / "host" / "dp")))
    assert nfiles >= 3
    assert compare_dirs(str(tmp_path / "host" / "dp"), str(tmp_path / "device" / "dp")) == []


_REPEAT = r"""
import sys, torch
sys.path.insert(0, sys.argv[1])
import idx2_b200
from idx2_b200.synthetic import grf_field_torch
out = sys.argv[2]
def field(seed, fronts):
    return grf_field_torch(512, 512, 512, seed=seed, scale="unit", n_fronts=fronts,
                           device=torch.device("cuda", 0)).cpu()
a = field(11, 20)
for d in sys.argv[3].split(","):
    which, tol, sub = d.split(":")
    f = a if which == "a" else field(12, 0)
    idx2_b200.encode(f, out_dir=out + "/" + sub, name="rp", field_name="f", num_levels=3, tolerance=float(tol))
    print("---", file=sys.stderr, flush=True)
"""


def _repeat(out_dir, plan):
    env = dict(os.environ, IDX2G_TRACE="1")
    r = subprocess.run([sys.executable, "-c", _REPEAT, ROOT, out_dir, plan], capture_output=True, text=True,
                       env=env, timeout=900)
    assert r.returncode == 0, r.stdout[-1000:] + r.stderr[-2000:]
    return r.stderr.split("---")


@pytest.mark.gpu
def test_repeated_encodes_with_premapped_files_equal_fresh_encodes(tmp_path):
    out = str(tmp_path)
    # one process: a, a into a new directory, a over the first files, then other fields whose
    # files are larger (tol 1e-4) and smaller (another seed at 1e-3) than the guess
    logs = _repeat(out, "a:1e-3:a1,a:1e-3:a2,a:1e-3:a1,a:1e-4:b1,b:1e-3:c1")
    assert "write.prealloc" not in logs[0], logs[0][-2000:]
    assert all("write.prealloc" in lg for lg in logs[1:5]), logs[1][-2000:]
    # fresh processes, one encode each
    _repeat(out, "a:1e-3:fa")
    _repeat(out, "a:1e-4:fb")
    _repeat(out, "b:1e-3:fc")
    big = max(os.path.getsize(os.path.join(dp, fn)) for dp, _, fs in os.walk(os.path.join(out, "fa", "rp")) for fn in fs)
    assert big >= 64 << 20  # (files from 64 MB on are allocated ahead)
    for got, want in (("a1", "fa"), ("a2", "fa"), ("b1", "fb"), ("c1", "fc")):
        assert compare_dirs(os.path.join(out, want, "rp"), os.path.join(out, got, "rp")) == [], got
