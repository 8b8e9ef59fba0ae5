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


@pytest.mark.gpu
def test_differentiable_decode_at_workload_sizes(idx2g, tmp_path):
    """The differentiable-decode workload's sizes: float32 fields of 256^3 (two of the batch of
    32; the fields of a batch are independent) and a float64 field of 128^3, 2 levels, seeded
    k^-5/3 fields encoded at tolerance 1e-4. D of the dataset's coefficients against the
    bit-exact decode; the float32 gradient of the MSE against the float64 adjoint of the same
    residual; the dot-product identity in both precisions; FP64 central differences at 20
    coefficients of the 128^3 field."""
    import torch
    from idx2_b200 import diff
    from idx2_b200.synthetic import grf_field_torch
    dev = torch.device("cuda", 0)

    def batch(n, side, dtype, seed):
        fmt = diff.Format((side, side, side), "float32" if dtype == torch.float32 else "float64", 2)
        cs, decs = [], []
        for i in range(n):
            f = grf_field_torch(side, side, side, seed=seed + i, scale="unit", device=dev).to(dtype)
            d = str(tmp_path / f"b{seed}_{i}")
            idx2g.encode(f, out_dir=d, name="adj", field_name="f", num_levels=2, tolerance=1e-4)
            ds = idx2g.Dataset(os.path.join(d, "adj", "f.idx2"))
            cs.append(diff.coefficients(ds, fmt, 1e-4))
            decs.append(torch.from_numpy(ds.decode(tolerance=1e-4)).to(dev))
            ds.close()
        return fmt, torch.stack(cs), torch.stack(decs)

    fmt, c, dec = batch(2, 256, torch.float32, 300)
    x = diff.synth(c, fmt)
    assert float((x - dec).abs().max() / dec.abs().max()) <= 1e-5
    target = torch.stack([grf_field_torch(256, 256, 256, seed=900 + i, scale="unit", device=dev) for i in range(2)])
    g32 = diff.synth_adjoint(2.0 * (x - target) / x.numel(), fmt)
    fmt64 = diff.Format(fmt.dims, "float64", 2)
    x64 = diff.synth(c.double(), fmt64)
    g64 = diff.synth_adjoint(2.0 * (x64 - target.double()) / x64.numel(), fmt64)
    assert float((g32.double() - g64).abs().max() / g64.abs().max()) <= 1e-5
    gen = torch.Generator(device=dev)
    gen.manual_seed(5)
    y = torch.randn(target.shape, generator=gen, device=dev, dtype=torch.float64)
    cd = torch.randn(c.shape, generator=gen, device=dev, dtype=torch.float64)
    lhs, rhs = float(torch.sum(diff.synth(cd, fmt64) * y)), float(torch.sum(cd * diff.synth_adjoint(y, fmt64)))
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs)
    lhs = float(torch.sum(diff.synth(cd.float(), fmt).double() * y))
    rhs = float(torch.sum(cd * diff.synth_adjoint(y.float(), fmt).double()))
    assert abs(lhs - rhs) <= 1e-4 * abs(lhs)
    del x, x64, g32, g64, y, cd, target, c, dec

    fmt_d, c_d, dec_d = batch(1, 128, torch.float64, 500)
    x = diff.synth(c_d, fmt_d)
    assert float((x - dec_d).abs().max() / dec_d.abs().max()) <= 1e-12
    target = grf_field_torch(128, 128, 128, seed=1900, scale="unit", device=dev).double()[None]
    grad = diff.synth_adjoint(2.0 * (x - target) / x.numel(), fmt_d)[0]
    c0 = c_d[0].clone()
    rng = np.random.default_rng(8)
    idx = [int(i) for i in rng.permutation(np.nonzero(grad.abs().cpu().numpy() > 0)[0])[:20]]
    h = 1e-3
    for i in idx:
        old = float(c0[i])
        c0[i] = old + h
        xp = diff.synth(c0, fmt_d)
        c0[i] = old - h
        xm = diff.synth(c0, fmt_d)
        c0[i] = old
        fd = float(torch.sum((xp - target[0]) ** 2 - (xm - target[0]) ** 2)) / x.numel() / (2 * h)
        assert abs(fd - float(grad[i])) <= 1e-6 * abs(fd) + 1e-14, (i, fd, float(grad[i]))
