"""CPU oracle for the Fourier-neural-operator surrogate.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``diffnano_b200``) imports
this module; only ``tests/`` use it, as the checker of the GPU operator's
forward values and parameter gradients.

Parity unpinned against the reference: DiffNano has no neural operator (its
surrogate is a small CNN, ``diffnano/solvers/surrogate.py:23-75``, trained
with mse_loss and Adam, ``:128, 193-197``), so there is no reference output to
pin.  This module restates the published 2-D Fourier neural operator (Li et
al., "Fourier Neural Operator for Parametric Partial Differential Equations",
ICLR 2021: lift, spectral convolution over the low rfft2 modes with complex
per-mode channel weights plus a pointwise linear path, GELU (tanh form), projection) with
the parameter layout of ``diffnano_b200.surrogate.fno`` and this project's
row readout, in FP32 with ``torch.fft.rfft2`` / ``irfft2`` on the CPU;
gradients come from torch autograd.  It shares no code with the GPU path: the
GPU computes the transforms as dense BF16 DFT-matrix GEMMs, the oracle with
FFTs.
"""

from __future__ import annotations

from typing import Dict

import torch
import torch.nn.functional as F


def features(eps: torch.Tensor, lo: float, hi: float) -> torch.Tensor:
    """(B, H, W) -> (B, H, W, 3): normalised eps, column and row coordinates."""
    B, H, W = eps.shape
    x = torch.linspace(0.0, 1.0, W, dtype=eps.dtype).view(1, 1, W).expand(B, H, W)
    y = torch.linspace(0.0, 1.0, H, dtype=eps.dtype).view(1, H, 1).expand(B, H, W)
    return torch.stack([(eps - lo) / (hi - lo), x, y], dim=-1)


def spectral(x: torch.Tensor, wre: torch.Tensor, wim: torch.Tensor, modes: int) -> torch.Tensor:
    """Spectral convolution of channel-last x (B, H, W, C) with complex
    weights w = wre + i*wim of shape (2*modes*modes, C_out, C_in), mode index
    m = khi*modes + kw; khi < modes are rows kh = khi, the rest kh = H - 2*modes
    + khi (the negative frequencies)."""
    B, H, W, C = x.shape
    xf = torch.fft.rfft2(x.permute(0, 3, 1, 2))  # (B, C, H, W//2+1)
    w = torch.complex(wre, wim).view(2 * modes, modes, wre.shape[1], wre.shape[2])
    out = torch.zeros(B, wre.shape[1], H, W // 2 + 1, dtype=xf.dtype)
    out[:, :, :modes, :modes] = torch.einsum("bixy,xyoi->boxy", xf[:, :, :modes, :modes],
                                             w[:modes])
    out[:, :, H - modes:, :modes] = torch.einsum("bixy,xyoi->boxy", xf[:, :, H - modes:, :modes],
                                                 w[modes:])
    return torch.fft.irfft2(out, s=(H, W)).permute(0, 2, 3, 1)


def forward(params: Dict[str, torch.Tensor], eps: torch.Tensor, *, layers: int, modes: int,
            n_out: int, lo: float, hi: float) -> torch.Tensor:
    """eps (B, H, W) -> prediction (B, W, n_out)."""
    f = features(eps, lo, hi)
    X = f @ params["P"][:, :3].T + params["p"]
    for l in range(layers):
        pre = spectral(X, params[f"wre{l}"], params[f"wim{l}"], modes) \
            + X @ params[f"W{l}"].T + params[f"b{l}"]
        X = F.gelu(pre, approximate="tanh") if l < layers - 1 else pre
    R = torch.einsum("bhwc,hc->bwc", X, params["r"])
    U = F.gelu(R @ params["Q1"].T + params["q1"], approximate="tanh")
    return U @ params["Q2"][:n_out].T + params["q2"][:n_out]


def loss_and_grads(params: Dict[str, torch.Tensor], eps: torch.Tensor, target: torch.Tensor,
                   **kw):
    """Mean squared error and its gradient with respect to every parameter
    (and to eps)."""
    ps = {k: v.detach().clone().requires_grad_(True) for k, v in params.items()}
    e = eps.detach().clone().requires_grad_(True)
    pred = forward(ps, e, **kw)
    loss = ((pred - target) ** 2).mean()
    loss.backward()
    return loss.detach(), pred.detach(), {k: v.grad for k, v in ps.items()}, e.grad
