"""Sharded encode through the C ABI on one GPU: the shards of one field run one after the other
in this process (each on its own context, the payload exchange done in memory), and the files
they write together equal the single-process encode's and the reference's. Covers the
device path of idx2g_encode_shard (shard plans on the GPU coder, fields given as each shard's
region only) that the gloo CPU test covers with the oracle's coder."""
import os
import subprocess

import numpy as np
import pytest

from idx2_files import compare_dirs

CASES = [
    ((256, 192, 128), "float32", 2, 1e-3, 2),
    ((256, 256, 256), "float32", 3, 1e-3, 4),
    ((160, 130, 100), "float64", 2, 1e-5, 3),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{c[1]}-L{c[2]}-s{c[4]}")
def test_shards_on_one_gpu_match_single_encode(idx2g, ref_app, tmp_path, case):
    import torch
    from idx2_b200.sharded import ShardEncode, shard_region
    from idx2_b200.synthetic import bumps_field
    dims, dt, levels, tol, n = case
    nx, ny, nz = dims
    f = bumps_field(nx, ny, nz, seed=51).astype(np.float32 if dt == "float32" else np.float64)
    full = torch.from_numpy(f).cuda()
    jobs = []
    for s in range(n):
        lo, sz = shard_region(dims, dt, levels, tol, s, n)
        # the shard's region only (a copy), as a process of a multi-GPU job would hold it
        region = full[lo[2]:lo[2] + sz[2], lo[1]:lo[1] + sz[1], lo[0]:lo[0] + sz[0]].contiguous()
        jobs.append(ShardEncode(region, lo, dims, str(tmp_path / "sharded"), "shd", "f", levels, tol, s, n,
                                own_context=True))
    payloads = [j.headers for j in jobs]
    vmin, vmax = min(j.vmin for j in jobs), max(j.vmax for j in jobs)
    for j in jobs:
        j.finish(payloads, vmin, vmax)
    idx2g.encode(f, out_dir=str(tmp_path / "single"), name="shd", field_name="f", num_levels=levels, tolerance=tol)
    assert compare_dirs(str(tmp_path / "single" / "shd"), str(tmp_path / "sharded" / "shd")) == []
    raw = str(tmp_path / f"shd-f-[{nx}-{ny}-{nz}]-{dt.capitalize()}.raw")
    f.tofile(raw)
    r = subprocess.run([ref_app, "--encode", raw, "--num_levels", str(levels), "--tolerance", repr(tol),
                        "--out_dir", str(tmp_path / "ref")], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-300:] + r.stderr[-300:]
    assert compare_dirs(str(tmp_path / "ref" / "shd"), str(tmp_path / "sharded" / "shd")) == []
    # every shard decodes its own region of the dataset; together they tile the field
    ds = idx2g.Dataset(str(tmp_path / "sharded" / "shd" / "f.idx2"))
    whole = ds.decode()
    for s in range(n):
        lo, sz = shard_region(dims, dt, levels, tol, s, n)
        part = ds.decode(first=lo, last=[lo[k] + sz[k] - 1 for k in range(3)])
        assert part.tobytes() == whole[lo[2]:lo[2] + sz[2], lo[1]:lo[1] + sz[1], lo[0]:lo[0] + sz[0]].tobytes()
    ds.close()
