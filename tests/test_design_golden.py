"""The design-layer oracle and the product's design operators against the
outputs of DiffNano's own operators (``tests/golden/design_ref.npz``, written
by ``tests/golden/make_design_golden.py`` from
``diffnano/design/projection.py:15-115``,
``diffnano/design/constraints_shared/primitives.py:27-66`` and
``diffnano/design/parameterization.py:248-300``).

CPU: the oracle (``oracle/design_ref.py``) reproduces every fixture bit for
bit -- Gaussian filter (3-D and 2-D inputs, seven radii), sigmoid projection,
``DensityField`` eps, the beta schedule, and the 3 x 3 erosion / dilation
through the reference's opening penalty and its gradient.  The product's
beta schedule (pure host code) matches too.  GPU: the product's FP32 kernels
against the same fixtures (relative L2 1e-6; morphology exact).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch
from conftest import GOLDEN, rel_l2

from oracle import design_ref as O

D = dict(np.load(f"{GOLDEN}/design_ref.npz"))
X3 = torch.tensor(D["x3"])
X2 = torch.tensor(D["x2"])
BLOBS = torch.tensor(D["blobs"])


def _opening_penalty(x, filt):
    """minimum_cd_penalty's arithmetic with erosion / dilation from ``filt``."""
    opened = filt.dilate(filt.erode(x))
    return ((x - opened) ** 2).mean()


@pytest.mark.parametrize("r", [float(v) for v in D["radii"]])
def test_oracle_smooth_filter_bit_exact(r):
    """Values bit for bit.  The reference returns an ``(N, 1, H, W)`` tensor
    for a batch of N > 1 maps (its squeeze logic keeps the channel axis,
    ``projection.py:78-83``); the oracle and the product return ``(N, H, W)``."""
    ref3 = D[f"smooth3_r{r}"]
    assert ref3.shape == (X3.shape[0], 1, *X3.shape[1:])
    assert np.array_equal(O.smooth_filter(X3, r).numpy(), ref3[:, 0])
    assert np.array_equal(O.smooth_filter(X2.unsqueeze(0), r)[0].numpy(), D[f"smooth2_r{r}"])


def test_oracle_projections_bit_exact():
    for b in D["betas"]:
        for e in D["etas"]:
            b, e = float(b), float(e)
            assert np.array_equal(O.heaviside_projection(X3, b, e).numpy(),
                                  D[f"heaviside_b{b}_e{e}"])
            eps = O.density_to_eps(X3[:1], 0.0, b, e, "sigmoid", 2.085, 12.1)[0]
            np.testing.assert_allclose(eps.numpy(), D[f"density_field_b{b}_e{e}"], rtol=0,
                                       atol=4e-15)


def test_beta_schedules_match_reference():
    from diffnano_b200.design.projection import beta_continuation_schedule

    got = [beta_continuation_schedule(int(s), int(n), b0, b1) for s, n, b0, b1 in
           D["schedule_args"]]
    assert np.array_equal(np.array(got), D["schedule"])


@pytest.mark.parametrize("name", ["x3", "blobs"])
@pytest.mark.parametrize("c", [float(v) for v in D["min_cd"]])
def test_oracle_erosion_dilation_through_reference_penalty(name, c):
    x = (X3 if name == "x3" else BLOBS).clone().requires_grad_(True)
    p = _opening_penalty(x, O)
    p.backward()
    assert float(p.detach()) == float(D[f"mincd_{name}_c{c}"])
    assert np.array_equal(x.grad.numpy(), D[f"mincd_grad_{name}_c{c}"])


@pytest.mark.gpu
def test_product_design_kernels_against_reference_outputs(cuda):
    from diffnano_b200.design import projection as P

    for r in [float(v) for v in D["radii"]]:
        got = P.smooth_filter(X3.float().to(cuda), r)
        assert rel_l2(got, D[f"smooth3_r{r}"][:, 0]) < 1e-6, r
    for b in D["betas"]:
        for e in D["etas"]:
            b, e = float(b), float(e)
            got = P.heaviside_projection(X3.float().to(cuda), b, e)
            assert rel_l2(got, D[f"heaviside_b{b}_e{e}"]) < 1e-6, (b, e)
            eps = P.density_to_eps(X3[:1].float().to(cuda), 0.0, b, e, "sigmoid", 2.085, 12.1)
            assert rel_l2(eps[0], D[f"density_field_b{b}_e{e}"]) < 1e-6, (b, e)
    for name, x0 in (("x3", X3), ("blobs", BLOBS)):
        x = x0.float().to(cuda).requires_grad_(True)
        p = _opening_penalty(x, P)
        p.backward()
        c = float(D["min_cd"][0])
        assert abs(float(p.detach()) / float(D[f"mincd_{name}_c{c}"]) - 1) < 1e-5
        assert rel_l2(x.grad, D[f"mincd_grad_{name}_c{c}"]) < 1e-5
