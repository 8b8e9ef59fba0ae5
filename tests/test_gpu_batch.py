"""Batched encode (idx2g_encode_batch): many uneven fields through one device stage must give,
field by field, the files of the single-field encode (which is itself checked against the
reference), with and without the CUDA graph, and with the device stage alone."""
import os
import subprocess

import numpy as np
import pytest

from idx2_files import compare_dirs


def _batch_fields(n, seed, max_side=110):
    import idx2_b200
    from idx2_b200.synthetic import bumps_field
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        dims = [int(rng.integers(17, max_side + 1)) for _ in range(3)]
        is2d = rng.integers(0, 8) == 0
        if is2d:
            dims[2] = 1
        dt = "float32" if rng.integers(0, 2) == 0 else "float64"
        levels = int(rng.integers(1, 4))
        bd = (32, 32, 1) if is2d else (32, 32, 32)
        p = idx2_b200.Params(dims=dims, dtype=dt, brick_dims=bd, num_levels=levels, tolerance=1e-3)
        if idx2_b200.check_params(p) != 0:
            continue  # rejected by the format rules (the reference rejects it too)
        f = bumps_field(dims[0], dims[1], dims[2], seed=int(rng.integers(1 << 30)))
        out.append((f.astype(np.float32 if dt == "float32" else np.float64), levels))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [True, False])
def test_batch_matches_single_field_encode(idx2g, tmp_path, graph):
    fields = _batch_fields(10, seed=21)
    names = [f"b{i}" for i in range(len(fields))]
    for (f, lv), nm in zip(fields, names):
        idx2g.encode(f, out_dir=str(tmp_path / "single"), name=nm, field_name="f", num_levels=lv,
                     tolerance=1e-3)
    infos = idx2g.encode_batch([f for f, _ in fields], out_dir=str(tmp_path / "batch"), names=names,
                               field_names=["f"] * len(fields), num_levels=[lv for _, lv in fields],
                               tolerances=[1e-3] * len(fields), graph=graph, autotune=True)
    assert len(infos) == len(fields)
    assert infos[0].kernel_launches == max(lv for _, lv in fields)  # one launch per level
    for nm in names:
        diffs = compare_dirs(str(tmp_path / "single" / nm), str(tmp_path / "batch" / nm))
        assert diffs == [], (nm, diffs[:3])


@pytest.mark.gpu
def test_batch_from_device_tensors_matches_reference(idx2g, ref_app, tmp_path):
    import torch
    fields = _batch_fields(6, seed=22, max_side=90)
    names = [f"d{i}" for i in range(len(fields))]
    idx2g.encode_batch([torch.from_numpy(f).cuda() for f, _ in fields], out_dir=str(tmp_path / "batch"),
                       names=names, field_names=["f"] * len(fields), num_levels=[lv for _, lv in fields],
                       tolerances=[1e-3] * len(fields))
    for (f, lv), nm in zip(fields, names):
        nz, ny, nx = f.shape if f.ndim == 3 else (1,) + f.shape
        dt = "Float32" if f.dtype == np.float32 else "Float64"
        raw = str(tmp_path / f"{nm}-f-[{nx}-{ny}-{nz}]-{dt}.raw")
        f.tofile(raw)
        args = [ref_app, "--encode", raw, "--num_levels", str(lv), "--tolerance", "0.001",
                "--out_dir", str(tmp_path / "ref")]
        if nz == 1:
            args += ["--brick_size", "32", "32", "1"]
        r = subprocess.run(args, capture_output=True, text=True)
        assert r.returncode == 0, r.stdout[-300:] + r.stderr[-300:]
        diffs = compare_dirs(str(tmp_path / "ref" / nm), str(tmp_path / "batch" / nm))
        assert diffs == [], (nm, diffs[:3])


@pytest.mark.gpu
def test_batch_device_only(idx2g, tmp_path):
    fields = _batch_fields(5, seed=23, max_side=80)
    infos = idx2g.encode_batch([f for f, _ in fields], out_dir=str(tmp_path / "none"),
                               num_levels=[lv for _, lv in fields], tolerances=[1e-3] * len(fields),
                               device_only=True)
    assert not os.path.exists(str(tmp_path / "none"))
    for (f, _), info in zip(fields, infos):
        assert info.value_min == pytest.approx(float(f.min()))
        assert info.value_max == pytest.approx(float(f.max()))


@pytest.mark.gpu
def test_batch_of_more_shapes_than_the_plan_cache(idx2g, tmp_path, monkeypatch):
    """A batch of more distinct field shapes than the context keeps plans for (a zero budget
    here, IDX2G_PLAN_CACHE_MB=0: each new plan drops the older ones): every field's plan stays
    valid for the whole call, the files match single-field encodes."""
    fields = _batch_fields(24, seed=33, max_side=48)
    assert len({f.shape + (lv,) for f, lv in fields}) > 16
    names = [f"m{i}" for i in range(len(fields))]
    for (f, lv), nm in zip(fields, names):
        idx2g.encode(f, out_dir=str(tmp_path / "single"), name=nm, field_name="f", num_levels=lv,
                     tolerance=1e-3)
    monkeypatch.setenv("IDX2G_PLAN_CACHE_MB", "0")
    idx2g.encode_batch([f for f, _ in fields], out_dir=str(tmp_path / "batch"), names=names,
                       field_names=["f"] * len(fields), num_levels=[lv for _, lv in fields],
                       tolerances=[1e-3] * len(fields), graph=True, autotune=False)
    monkeypatch.delenv("IDX2G_PLAN_CACHE_MB")
    for nm in names:
        diffs = compare_dirs(str(tmp_path / "single" / nm), str(tmp_path / "batch" / nm))
        assert diffs == [], (nm, diffs[:3])


@pytest.mark.gpu
def test_uneven_batch_of_64_fields_matches_reference(idx2g, ref_app, tmp_path):
    """The uneven-field workload at scale: 64 accepted fields drawn like the batched-encode
    benchmark (k^-5/3 Gaussian random fields scaled to [-1, 1], each axis 17-300, 1 in 8 2D,
    float32 and float64 alternating, levels 1-3, tolerance 1e-3) in one batched call; every
    field's files equal the reference CLI's encode of that field."""
    import torch
    from concurrent.futures import ThreadPoolExecutor
    from idx2_b200.synthetic import grf_field_torch
    rng = np.random.default_rng(77)
    fields, params = [], []
    i = 0
    while len(fields) < 64:
        dims = [int(rng.integers(17, 301)) for _ in range(3)]
        if rng.integers(0, 8) == 0:
            dims[2] = 1
        dt = "float32" if i % 2 == 0 else "float64"
        lv = int(rng.integers(1, 4))
        bd = (32, 32, 1) if dims[2] == 1 else (32, 32, 32)
        i += 1
        if idx2g.check_params(idx2g.Params(dims=dims, dtype=dt, brick_dims=bd, num_levels=lv, tolerance=1e-3)):
            continue
        f = grf_field_torch(dims[0], dims[1], dims[2], seed=9000 + i, scale="range", device=torch.device("cuda", 0))
        fields.append(f.to(torch.float32 if dt == "float32" else torch.float64).contiguous())
        params.append((dims, dt, lv))
    assert {p[1] for p in params} == {"float32", "float64"} and any(p[0][2] == 1 for p in params)
    names = [f"u{k}" for k in range(len(fields))]
    idx2g.encode_batch(fields, out_dir=str(tmp_path / "batch"), names=names, field_names=["f"] * len(fields),
                       num_levels=[p[2] for p in params], tolerances=[1e-3] * len(fields), graph=True,
                       autotune=True)

    def ref_one(k):
        (nx, ny, nz), dt, lv = params[k]
        raw = str(tmp_path / f"{names[k]}-f-[{nx}-{ny}-{nz}]-{dt.capitalize()}.raw")
        fields[k].cpu().numpy().tofile(raw)
        args = [ref_app, "--encode", raw, "--num_levels", str(lv), "--tolerance", "0.001",
                "--out_dir", str(tmp_path / "ref")]
        if nz == 1:
            args += ["--brick_size", "32", "32", "1"]
        r = subprocess.run(args, capture_output=True, text=True)
        os.remove(raw)
        return r.returncode, r.stdout[-300:] + r.stderr[-300:]

    with ThreadPoolExecutor(max_workers=max(1, min(16, os.cpu_count() or 1))) as pool:
        results = list(pool.map(ref_one, range(len(fields))))
    for k, (rc, msg) in enumerate(results):
        assert rc == 0, (names[k], msg)
        diffs = compare_dirs(str(tmp_path / "ref" / names[k]), str(tmp_path / "batch" / names[k]))
        assert diffs == [], (names[k], params[k], diffs[:3])
