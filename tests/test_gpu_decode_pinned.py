"""Decodes into pinned host memory (the output level runs in bands of brick rows whose finished
output planes go to the host while the next bands decode) give the bytes of the decode into
device memory, which the other decode tests check against the reference decoder."""
import numpy as np
import pytest

CASES = [
    # dims (x, y, z), dtype, levels, request (first, last, downsampling, tolerance)
    ((256, 256, 256), "float32", 3, (None, None, (0, 0, 0), 0.0)),
    ((256, 256, 256), "float32", 3, ((0, 0, 37), (255, 255, 250), (0, 0, 0), 0.0)),
    ((256, 256, 256), "float32", 2, (None, None, (0, 0, 0), 1e-2)),
    ((208, 200, 256), "float64", 2, (None, None, (0, 0, 0), 0.0)),
    ((208, 200, 256), "float64", 2, ((5, 0, 11), (207, 190, 255), (0, 0, 0), 0.0)),
    ((256, 256, 256), "float32", 3, (None, None, (1, 1, 1), 0.0)),
    ((256, 256, 256), "float32", 3, ((3, 9, 40), (250, 255, 255), (0, 1, 0), 0.0)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("ci", range(len(CASES)))
def test_pinned_host_decode_matches_device_decode(idx2g, tmp_path, ci):
    import torch
    from idx2_b200.synthetic import bumps_field
    dims, dt, levels, (first, last, down, tol) = CASES[ci]
    f = bumps_field(dims[0], dims[1], dims[2], seed=40 + ci).astype(np.float32 if dt == "float32" else np.float64)
    idx2g.encode(f, out_dir=str(tmp_path), name="p", field_name="f", num_levels=levels, tolerance=1e-4)
    ds = idx2g.Dataset(str(tmp_path / "p" / "f.idx2"))
    _, od, _ = ds.output_grid(first, last, down)
    shape = (od[2], od[1], od[0])
    tdt = torch.float32 if dt == "float32" else torch.float64
    dev = torch.empty(shape, dtype=tdt, device="cuda")
    ds.decode(first=first, last=last, downsampling=down, tolerance=tol, out=dev)
    host = torch.full(shape, float("nan"), dtype=tdt).pin_memory()
    assert host.numel() * host.element_size() >= 8 << 20
    ds.decode(first=first, last=last, downsampling=down, tolerance=tol, out=host)
    again = torch.full(shape, float("nan"), dtype=tdt).pin_memory()
    ds.decode(first=first, last=last, downsampling=down, tolerance=tol, out=again)
    ds.close()
    assert torch.equal(dev.cpu(), host)
    assert torch.equal(host, again)
