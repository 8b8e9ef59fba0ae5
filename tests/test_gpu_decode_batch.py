"""Batched decode (idx2g_decode_batch) and the serving layer on the GPU: every request of a
batch (its own extent, downsampling and tolerance) must equal the same request decoded alone,
bit for bit; the one-at-a-time decode is itself checked against the reference."""
import os

import numpy as np
import pytest


def _requests(dims, n, seed, is2d=False):
    rng = np.random.default_rng(seed)
    out = [{}]  # the whole field at full resolution
    for _ in range(n):
        first, last = [], []
        for a in range(3):
            d = dims[a]
            if d == 1:
                first.append(0)
                last.append(0)
                continue
            s = int(rng.integers(1, d + 1))
            f = int(rng.integers(0, d - s + 1))
            first.append(f)
            last.append(f + s - 1)
        ds = tuple(int(rng.integers(0, 3)) if dims[a] > 1 else 0 for a in range(3))
        tol = [0.0, 1e-3, 1e-2, 1e-1][int(rng.integers(0, 4))]
        out.append({"first": tuple(first), "last": tuple(last), "downsampling": ds, "tolerance": tol})
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("dims,dtype,levels", [((160, 128, 96), np.float32, 2), ((200, 150, 1), np.float64, 2)])
def test_decode_batch_equals_single_requests(idx2g, tmp_path, dims, dtype, levels):
    import torch
    from idx2_b200.synthetic import bumps_field
    f = bumps_field(dims[0], dims[1], dims[2], seed=5).astype(dtype)
    idx2g.encode(f, out_dir=str(tmp_path), name="kat", field_name="f", num_levels=levels, tolerance=1e-4)
    ds = idx2g.Dataset(os.path.join(str(tmp_path), "kat", "f.idx2"))
    reqs = _requests(dims, 24, seed=9)
    outs = ds.decode_batch(reqs, device_out=True)
    assert len(outs) == len(reqs)
    for r, o in zip(reqs, outs):
        _, odims, _ = ds.output_grid(r.get("first"), r.get("last"), r.get("downsampling", (0, 0, 0)))
        single = torch.empty((odims[2], odims[1], odims[0]), dtype=o.dtype, device=o.device)
        ds.decode(r.get("first"), r.get("last"), r.get("downsampling", (0, 0, 0)), r.get("tolerance", 0.0),
                  out=single)
        assert torch.equal(single, o), r
    host = ds.decode_batch(reqs[:5], device_out=False)
    for h, o in zip(host, outs[:5]):
        assert np.array_equal(h, o.cpu().numpy())
    ds.close()


@pytest.mark.gpu
def test_serving_run(idx2g, tmp_path):
    from idx2_b200.synthetic import bumps_field
    from idx2_b200.serving import Server, dataset_decoder, poisson_schedule, free_hbm_budget
    dims = (192, 160, 128)  # 2 levels (3 would break the format's level rule for these dims)
    f = bumps_field(*dims, seed=6).astype(np.float32)
    idx2g.encode(f, out_dir=str(tmp_path), name="srv", field_name="f", num_levels=2, tolerance=1e-5)
    ds = idx2g.Dataset(os.path.join(str(tmp_path), "srv", "f.idx2"))
    sched = poisson_schedule(60, 2000.0, dims, seed=4, side=(16, 96))
    budget = min(free_hbm_budget(), 2 << 30)
    srv = Server(dataset_decoder(ds), budget)
    st = srv.run([r for r in sched], batched=True)
    assert st.requests + st.rejected == 60 and st.rejected == 0
    assert st.batches < 60 and st.p99_ms >= st.p50_ms > 0
    ds.close()
