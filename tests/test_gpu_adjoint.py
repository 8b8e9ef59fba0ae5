"""Differentiable decode on the GPU: the real-valued decode operator D (idx2g_synth) against the
FP64 torch reference, its adjoint kernel (idx2g_synth_adjoint) through the dot-product identity,
gradients through the autograd Function against the FP64 reference gradient and FP64 central
finite differences, and D applied to a dataset's dequantised coefficients against the bit-exact
decode."""
import os

import numpy as np
import pytest

import synth_reference as ref

CASES = [((70, 66, 65), 2), ((200, 150, 1), 2), ((100, 90, 70), 2)]


def _coeffs(n, seed, dtype, device="cuda"):
    import torch
    g = torch.Generator().manual_seed(seed)
    return torch.randn(n, generator=g, dtype=torch.float64).to(device=device, dtype=dtype)


@pytest.mark.gpu
@pytest.mark.parametrize("dims,levels", CASES)
def test_synth_matches_fp64_reference(idx2g, dims, levels):
    import torch
    from idx2_b200.diff import Format, coeff_count, synth
    fmt = Format(dims, "float64", levels)
    c = _coeffs(coeff_count(fmt), 1, torch.float64)
    got = synth(c, fmt).cpu()
    want = ref.synth(c.cpu(), dims, levels)
    assert torch.allclose(got, want, rtol=1e-12, atol=1e-12 * float(want.abs().max()))


@pytest.mark.gpu
@pytest.mark.parametrize("dims,levels", CASES)
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_adjoint_dot_product(idx2g, dims, levels, dtype):
    import torch
    from idx2_b200.diff import Format, coeff_count, synth, synth_adjoint
    fmt = Format(dims, dtype, levels)
    td = torch.float64 if dtype == "float64" else torch.float32
    c = _coeffs(coeff_count(fmt), 2, td)
    g = _coeffs(int(np.prod(dims)), 3, td).reshape(fmt.shape)
    lhs = float((synth(c, fmt).double() * g.double()).sum())
    rhs = float((c.double() * synth_adjoint(g, fmt).double()).sum())
    tol = 1e-11 if dtype == "float64" else 1e-4
    assert abs(lhs - rhs) <= tol * max(abs(lhs), 1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("dims,levels", CASES)
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_gradient_matches_fp64_reference(idx2g, dims, levels, dtype):
    import torch
    from idx2_b200.diff import Format, coeff_count, decode_diff
    fmt = Format(dims, dtype, levels)
    td = torch.float64 if dtype == "float64" else torch.float32
    n = coeff_count(fmt)
    c0 = _coeffs(n, 4, torch.float64, device="cpu")
    target = _coeffs(int(np.prod(dims)), 5, torch.float64, device="cpu").reshape(fmt.shape)
    # FP64 reference gradient of the MSE loss
    cr = c0.clone().requires_grad_(True)
    torch.mean((ref.synth(cr, dims, levels) - target) ** 2).backward()
    want = cr.grad
    # through the autograd Function (hand-written adjoint kernel)
    c = c0.to(device="cuda", dtype=td).requires_grad_(True)
    loss = torch.mean((decode_diff(c, fmt) - target.to(device="cuda", dtype=td)) ** 2)
    loss.backward()
    got = c.grad.double().cpu()
    rel = float((got - want).norm() / want.norm())
    assert rel <= (1e-10 if dtype == "float64" else 1e-5), rel


@pytest.mark.gpu
def test_gradient_matches_central_differences(idx2g):
    import torch
    from idx2_b200.diff import Format, coeff_count, decode_diff, synth
    dims, levels = (100, 90, 70), 2
    fmt = Format(dims, "float64", levels)
    n = coeff_count(fmt)
    c = _coeffs(n, 6, torch.float64).requires_grad_(True)
    target = _coeffs(int(np.prod(dims)), 7, torch.float64).reshape(fmt.shape)
    loss = torch.mean((decode_diff(c, fmt) - target) ** 2)
    loss.backward()
    grad = c.grad.detach()
    # 200 random coefficients that the grid depends on (gradient not zero), step 1e-3. The
    # difference of the two losses is summed sample by sample: samples outside the coefficient's
    # support cancel exactly, so the rounding error scales with the support, not the whole loss
    # (the loss is quadratic in c: the central difference itself has no truncation error).
    rng = np.random.default_rng(8)
    idx = [int(i) for i in rng.permutation(np.nonzero(grad.abs().cpu().numpy() > 0)[0])[:200]]
    h = 1e-3
    cd = c.detach().clone()
    for i in idx:
        old = float(cd[i])
        cd[i] = old + h
        xp = synth(cd, fmt)
        cd[i] = old - h
        xm = synth(cd, fmt)
        cd[i] = old
        fd = float(torch.sum((xp - target) ** 2 - (xm - target) ** 2)) / target.numel() / (2 * h)
        assert abs(fd - float(grad[i])) <= 1e-6 * abs(fd) + 1e-14, (i, fd, float(grad[i]))


@pytest.mark.gpu
@pytest.mark.parametrize("dims,dtype", [((100, 90, 70), "float64"), ((200, 150, 1), "float32")])
def test_synth_of_dataset_coefficients_matches_decode(idx2g, tmp_path, dims, dtype):
    import torch
    from idx2_b200.diff import Format, coefficients, synth
    from idx2_b200.synthetic import bumps_field
    f = bumps_field(*dims, seed=12).astype(np.float32 if dtype == "float32" else np.float64)
    idx2g.encode(f, out_dir=str(tmp_path), name="d", field_name="f", num_levels=2, tolerance=1e-4)
    ds = idx2g.Dataset(os.path.join(str(tmp_path), "d", "f.idx2"))
    fmt = Format(dims, dtype, 2)
    c = coefficients(ds, fmt)
    x = synth(c, fmt)
    dec = ds.decode()
    xd = x.cpu().numpy().reshape(dec.shape)
    # D differs from the bit-exact decode only by the floors of the integer inverse zfp
    # (and float32 rounding for float32 data); every low-band block of these fields is decoded,
    # so in 2D no block keeps the parent's values
    scale = float(np.abs(dec).max())
    tol = 1e-12 if dtype == "float64" else 1e-5
    assert float(np.abs(xd - dec).max()) <= tol * scale
    ds.close()
