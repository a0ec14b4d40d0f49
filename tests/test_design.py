"""Design-layer kernels (density filter, sigmoid / tanh projection, erosion /
dilation) against the CPU oracle of the reference's operators: values and
gradients."""

from __future__ import annotations

import pytest
import torch

from oracle import design_ref

from conftest import rel_l2


def test_beta_schedule_matches_reference_formula():
    from diffnano_b200.design.projection import beta_continuation_schedule as b
    assert b(0, 100, 1.0, 32.0) == 1.0
    assert abs(b(100, 100, 1.0, 32.0) - 32.0) < 1e-12
    assert abs(b(50, 100, 1.0, 64.0) - 8.0) < 1e-12
    assert b(500, 100, 1.0, 32.0) == b(100, 100, 1.0, 32.0)


@pytest.mark.gpu
@pytest.mark.parametrize("projection,radius,beta", [("tanh", 4.0, 8.0), ("sigmoid", 2.0, 3.0),
                                                    ("none", 6.0, 1.0), ("tanh", 0.0, 32.0)])
def test_density_to_eps_values_and_gradient(cuda, projection, radius, beta):
    from diffnano_b200.design.projection import density_to_eps
    g = torch.Generator().manual_seed(1)
    rho = torch.rand(5, 40, 67, generator=g, dtype=torch.float32)
    w = torch.randn(5, 40, 67, generator=g, dtype=torch.float32)
    x = rho.clone().requires_grad_(True)
    ref = design_ref.density_to_eps(x.double(), radius, beta, 0.5, projection, 2.085, 12.1)
    (ref * w.double()).sum().backward()
    xd = rho.to(cuda).requires_grad_(True)
    out = density_to_eps(xd, radius, beta, 0.5, projection, 2.085, 12.1)
    (out * w.to(cuda)).sum().backward()
    assert rel_l2(out, ref) < 1e-6
    assert rel_l2(xd.grad, x.grad) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("op", ["erode", "dilate"])
def test_morphology_matches_max_pool(cuda, op):
    from diffnano_b200.design import projection as P
    g = torch.Generator().manual_seed(2)
    # binary maps (many ties) and continuous ones
    for x0 in ((torch.rand(3, 33, 50, generator=g) > 0.5).float(), torch.rand(3, 33, 50, generator=g)):
        w = torch.randn(x0.shape, generator=g)
        x = x0.clone().requires_grad_(True)
        ref = getattr(design_ref, op)(x)
        (ref * w).sum().backward()
        xd = x0.to(cuda).requires_grad_(True)
        out = getattr(P, op)(xd)
        (out * w.to(cuda)).sum().backward()
        assert torch.equal(out.cpu(), ref.detach())
        assert rel_l2(xd.grad, x.grad) < 1e-6
