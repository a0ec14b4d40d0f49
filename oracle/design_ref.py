"""CPU oracle for the design-layer kernels (density -> permittivity).

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module; only
``tests/`` use it as the checker of ``diffnano_b200.design.projection``.

Restates DiffNano's design-layer operators in torch on the CPU, following the
reference line by line in meaning:

* ``smooth_filter`` -- ``diffnano/design/projection.py:39-85``: 1-D Gaussian
  taps ``exp(-x^2 / (2 sigma^2 + 1e-12))`` over ``k = int(2r+1)`` (made odd)
  points, sigma = r/2, normalised, outer product, ``conv2d`` with zero
  padding ``(k-1)/2``; applied here to every layer of an ``(L, H, W)`` field;
* ``heaviside_projection`` -- ``projection.py:15-36``: ``sigmoid(beta (x - eta))``;
* ``tanh_projection`` -- the tanh projection (an addition: not in the reference);
* ``erode`` / ``dilate`` -- ``diffnano/design/constraints_shared/primitives.py:56-60``:
  ``-max_pool2d(-x, 3, 1, 1)`` / ``max_pool2d(x, 3, 1, 1)``.

Gradients come from torch autograd.
"""
from __future__ import annotations

import torch
import torch.nn.functional as F


def smooth_filter(x: torch.Tensor, radius: float) -> torch.Tensor:
    """(L, H, W) -> (L, H, W)."""
    k = int(2 * radius + 1)
    if k % 2 == 0:
        k += 1
    sigma = radius / 2.0
    t = torch.arange(k, dtype=x.dtype) - k // 2
    g = torch.exp(-(t ** 2) / (2 * sigma ** 2 + 1e-12))
    g = g / g.sum()
    ker = (g.unsqueeze(1) @ g.unsqueeze(0)).view(1, 1, k, k)
    return F.conv2d(x.unsqueeze(1), ker, padding=(k - 1) // 2)[:, 0]


def heaviside_projection(x: torch.Tensor, beta: float, eta: float = 0.5) -> torch.Tensor:
    return torch.sigmoid(beta * (x - eta))


def tanh_projection(x: torch.Tensor, beta: float, eta: float = 0.5) -> torch.Tensor:
    a = torch.tanh(torch.tensor(beta * eta, dtype=x.dtype))
    b = torch.tanh(torch.tensor(beta * (1 - eta), dtype=x.dtype))
    return (a + torch.tanh(beta * (x - eta))) / (a + b)


def density_to_eps(rho, radius, beta, eta, projection, lo, hi):
    xf = smooth_filter(rho, radius)
    if projection == "sigmoid":
        p = heaviside_projection(xf, beta, eta)
    elif projection == "tanh":
        p = tanh_projection(xf, beta, eta)
    else:
        p = xf
    return lo + (hi - lo) * p


def erode(x: torch.Tensor) -> torch.Tensor:
    return -F.max_pool2d(-x.unsqueeze(1), 3, 1, 1)[:, 0]


def dilate(x: torch.Tensor) -> torch.Tensor:
    return F.max_pool2d(x.unsqueeze(1), 3, 1, 1)[:, 0]
