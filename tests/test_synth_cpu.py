"""Differentiable decode, host side (no GPU): the coefficient tensor's length from the library
matches the layout the FP64 reference assumes, and the reference operator is linear."""
import pytest
import torch

import synth_reference as ref


@pytest.mark.parametrize("dims,levels", [((70, 66, 65), 2), ((100, 90, 70), 2), ((200, 150, 1), 2), ((256, 256, 1), 3)])
def test_coeff_count_matches_reference_layout(dims, levels):
    from idx2_b200.diff import Format, coeff_count
    assert coeff_count(Format(dims, "float64", levels)) == ref.coeff_count(dims, levels)


def test_reference_operator_is_linear():
    dims, levels = (40, 36, 34), 2
    n = ref.coeff_count(dims, levels)
    g = torch.Generator().manual_seed(0)
    a = torch.randn(n, generator=g, dtype=torch.float64)
    b = torch.randn(n, generator=g, dtype=torch.float64)
    lhs = ref.synth(2.0 * a - 3.0 * b, dims, levels)
    rhs = 2.0 * ref.synth(a, dims, levels) - 3.0 * ref.synth(b, dims, levels)
    assert torch.allclose(lhs, rhs, rtol=1e-12, atol=1e-12)
