"""Seeded synthetic permittivity maps and sources for the benchmark workloads.

These are host-side set-up helpers (not timed).  The filters restate
DiffNano's design-layer operators:

* ``smooth_filter`` -- Gaussian blur, ``diffnano/design/projection.py:39-85``
  (kernel size 2r+1 forced odd, sigma = r/2, zero padding);
* ``erode`` / ``dilate`` -- ``-max_pool2d(-x, 3, 1, 1)`` / ``max_pool2d(x, 3, 1, 1)``,
  ``diffnano/design/constraints_shared/primitives.py:56-60``.

Workloads (all seeded, all CPU FP64 on construction):

* ``blob_eps_2d`` -- 2-D SiO2 background (2.085) with a central Si (12.1) /
  SiO2 binary-blob design region from thresholded, Gaussian-filtered N(0,1)
  noise (the 256x256 TMz workload and the batched instances);
* ``slab_eps_3d`` -- 3-D air / 500 nm Si slab / SiO2 substrate stack with a
  design block of continuous eps in [2.085, 12.1] from filtered uniform noise
  (the 256^3 forward + adjoint workload).
"""

from __future__ import annotations

import math

import torch
import torch.nn.functional as F

EPS_SIO2 = 2.085
EPS_SI = 12.1
EPS_AIR = 1.0


def gaussian_pulse_for_band(center_nm: float, bandwidth_nm: float, amplitude: float = 1.0):
    """Reference-style source dict for a pulse of the given spectral width.

    The reference's pulse is ``sin(w t) exp(-(t-t0)^2 / (2 spread^2))`` with
    ``w = 2 pi / lambda`` (c = 1, nm units).  A spectral 1-sigma width
    ``d_lambda`` maps to ``spread = lambda^2 / (2 pi d_lambda)``; ``t0`` is
    three spreads so the pulse starts from ~0.
    """
    spread = center_nm ** 2 / (2.0 * math.pi * bandwidth_nm)
    return {"type": "gaussian_pulse", "spread": spread, "t0": 3.0 * spread,
            "amplitude": amplitude}


def smooth_filter(x: torch.Tensor, radius: float) -> torch.Tensor:
    """Gaussian blur of a ``(H, W)`` or ``(N, H, W)`` map (projection.py:39-85)."""
    squeeze = x.dim() == 2
    if squeeze:
        x = x.unsqueeze(0)
    x = x.unsqueeze(1)
    k = int(2 * radius + 1)
    if k % 2 == 0:
        k += 1
    sigma = radius / 2.0
    t = torch.arange(k, dtype=x.dtype) - k // 2
    g = torch.exp(-(t ** 2) / (2 * sigma ** 2 + 1e-12))
    g = g / g.sum()
    ker = (g.unsqueeze(1) @ g.unsqueeze(0)).view(1, 1, k, k)
    y = F.conv2d(x, ker, padding=(k - 1) // 2)[:, 0]
    return y[0] if squeeze else y


def erode(mask: torch.Tensor) -> torch.Tensor:
    """One-cell erosion of a 0/1 map (primitives.py:56-60)."""
    return -F.max_pool2d(-mask.unsqueeze(0).unsqueeze(0), 3, 1, 1)[0, 0]


def dilate(mask: torch.Tensor) -> torch.Tensor:
    """One-cell dilation of a 0/1 map (primitives.py:56-60)."""
    return F.max_pool2d(mask.unsqueeze(0).unsqueeze(0), 3, 1, 1)[0, 0]


def blob_design(n: int, seed: int, sigma_cells: float = 3.0) -> torch.Tensor:
    """``n x n`` 0/1 FP64 blob map: N(0,1) noise, Gaussian sigma, threshold 0.

    ``smooth_filter`` takes a radius with sigma = radius/2, so a sigma of 3
    cells is radius 6 (13-tap kernel).
    """
    g = torch.Generator().manual_seed(seed)
    noise = torch.randn(n, n, dtype=torch.float64, generator=g)
    return (smooth_filter(noise, 2.0 * sigma_cells) > 0).to(torch.float64)


def blob_eps_2d(side: int = 256, design: int = 128, seed: int = 0,
                sigma_cells: float = 3.0, variant: int = 0) -> torch.Tensor:
    """2-D eps map: SiO2 background, central ``design`` square of Si/SiO2 blobs.

    ``variant`` -1 / 0 / +1 applies a one-cell erosion / nothing / dilation to
    the blob mask (robust-design variants).
    """
    m = blob_design(design, seed, sigma_cells)
    if variant < 0:
        m = erode(m)
    elif variant > 0:
        m = dilate(m)
    eps = torch.full((side, side), EPS_SIO2, dtype=torch.float64)
    o = (side - design) // 2
    eps[o:o + design, o:o + design] = EPS_SIO2 + (EPS_SI - EPS_SIO2) * m
    return eps


def slab_eps_3d(shape=(256, 256, 256), dl: float = 25.0, slab_nm: float = 500.0,
                substrate_cells: int | None = None, design=(40, 128, 128), seed: int = 1,
                radius: float = 4.0) -> torch.Tensor:
    """3-D eps (z = axis 0): SiO2 substrate, Si slab, air above, design block.

    The slab is ``round(slab_nm/dl)`` cells thick starting at
    ``substrate_cells`` (default D*3/8).  The design block
    ``(dz, dy, dx)`` sits centred in x, y, starting at the slab's bottom; it
    is filled with ``2.085 + (12.1-2.085)*u`` where ``u`` is seeded U(0,1)
    noise blurred in-plane and min-max normalised to [0, 1].
    """
    D, H, W = shape
    eps = torch.full((D, H, W), EPS_AIR, dtype=torch.float64)
    z0 = substrate_cells if substrate_cells is not None else (3 * D) // 8
    t = int(round(slab_nm / dl))
    eps[:z0] = EPS_SIO2
    eps[z0:z0 + t] = EPS_SI
    dz, dy, dx = design
    g = torch.Generator().manual_seed(seed)
    u = torch.rand(dz, dy, dx, dtype=torch.float64, generator=g)
    u = smooth_filter(u, radius)
    u = (u - u.min()) / (u.max() - u.min() + 1e-30)
    y0, x0 = (H - dy) // 2, (W - dx) // 2
    eps[z0:z0 + dz, y0:y0 + dy, x0:x0 + dx] = EPS_SIO2 + (EPS_SI - EPS_SIO2) * u
    return eps
