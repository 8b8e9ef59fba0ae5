"""Encodes of a field in pinned host memory (copied in bands of brick rows on a second stream
while level 0's launches run) write the files of the encode of the same field from pageable
host memory and from device memory, which the other encode tests check against the reference
encoder."""
import numpy as np
import pytest

from idx2_files import compare_dirs

CASES = [
    # dims (x, y, z), dtype, levels, tolerance
    ((256, 192, 160), "float32", 3, 1e-3),
    ((100, 90, 75), "float64", 2, 1e-5),
    ((64, 64, 300), "float32", 1, 1e-4),
    ((65, 66, 97), "float64", 2, 1e-3),
    ((33, 40, 97), "float32", 1, 1e-3),
]


@pytest.mark.gpu
@pytest.mark.parametrize("ci", range(len(CASES)))
def test_pinned_host_encode_matches(idx2g, tmp_path, ci):
    import torch
    from idx2_b200.synthetic import bumps_field
    dims, dt, levels, tol = CASES[ci]
    f = bumps_field(dims[0], dims[1], dims[2], seed=70 + ci).astype(np.float32 if dt == "float32" else np.float64)
    kw = dict(field_name="f", num_levels=levels, tolerance=tol)
    idx2g.encode(f, out_dir=str(tmp_path / "pageable"), name="e", **kw)
    idx2g.encode(torch.from_numpy(f).cuda(), out_dir=str(tmp_path / "device"), name="e", **kw)
    pinned = torch.from_numpy(f).pin_memory()
    for rep in range(2):
        idx2g.encode(pinned, out_dir=str(tmp_path / f"pinned{rep}"), name="e", **kw)
    for other in ("device", "pinned0", "pinned1"):
        diffs = compare_dirs(str(tmp_path / "pageable" / "e"), str(tmp_path / other / "e"))
        assert diffs == [], (other, diffs[:3])


@pytest.mark.gpu
def test_device_field_off_16_byte_alignment(idx2g, tmp_path):
    """A device field that starts 4 bytes past a 16-byte boundary (a view into a larger
    tensor) cannot be read through a tensor map: the gather falls back to ordinary copies and
    the files are the same."""
    import torch
    from idx2_b200.synthetic import bumps_field
    dims = (128, 96, 80)
    f = bumps_field(dims[0], dims[1], dims[2], seed=90).astype(np.float32)
    kw = dict(field_name="f", num_levels=2, tolerance=1e-4)
    idx2g.encode(f, out_dir=str(tmp_path / "aligned"), name="e", **kw)
    big = torch.empty(f.size + 1, dtype=torch.float32, device="cuda")
    view = big[1:].view(dims[2], dims[1], dims[0])
    view.copy_(torch.from_numpy(f))
    assert view.data_ptr() % 16 == 4
    idx2g.encode(view, out_dir=str(tmp_path / "offset"), name="e", **kw)
    diffs = compare_dirs(str(tmp_path / "aligned" / "e"), str(tmp_path / "offset" / "e"))
    assert diffs == [], diffs[:3]
