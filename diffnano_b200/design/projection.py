"""Differentiable density -> permittivity pipeline on the GPU.

Restates DiffNano's design-layer operators as CUDA kernels
(``include/dn_design.h``):

* ``smooth_filter`` -- Gaussian blur, ``diffnano/design/projection.py:39-85``
  (kernel 2r+1 made odd, sigma = r/2, zero padding), applied in every layer;
* ``heaviside_projection`` -- ``sigmoid(beta (x - eta))``, ``projection.py:15-36``;
* ``tanh_projection`` -- the tanh projection
  ``(tanh(beta eta) + tanh(beta (x - eta))) / (tanh(beta eta) + tanh(beta (1 - eta)))``
  (an addition: the reference projects with a sigmoid only);
* ``beta_continuation_schedule`` -- ``projection.py:88-115`` (same formula);
* ``erode`` / ``dilate`` -- ``-max_pool2d(-x, 3, 1, 1)`` / ``max_pool2d(x, 3, 1, 1)``,
  ``diffnano/design/constraints_shared/primitives.py:56-60``.

``density_to_eps`` fuses filter, projection and the affine map to eps in one
forward call and one backward call.  All inputs are FP32 CUDA tensors of shape
``(H, W)`` or ``(L, H, W)`` (L layers filtered independently); there is no CPU
path.
"""
from __future__ import annotations

import ctypes

import torch

from .. import _lib

KINDS = {"sigmoid": 0, "tanh": 1, "none": 2}


def _as_layers(x: torch.Tensor) -> torch.Tensor:
    if not x.is_cuda:
        raise ValueError("the density pipeline runs on CUDA tensors")
    if x.dim() == 2:
        x = x.unsqueeze(0)
    if x.dim() != 3:
        raise ValueError(f"density must be (H, W) or (L, H, W), got {tuple(x.shape)}")
    return x.to(torch.float32).contiguous()


def _desc(x: torch.Tensor, radius, beta, eta, kind, lo, hi) -> _lib.DnDensity:
    L, H, W = x.shape
    return _lib.DnDensity(L, H, W, KINDS[kind], float(radius), float(beta), float(eta),
                          float(lo), float(hi))


class _DensityToEps(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rho, radius, beta, eta, kind, lo, hi):
        shape = rho.shape
        x = _as_layers(rho)
        d = _desc(x, radius, beta, eta, kind, lo, hi)
        work, filt, eps = (torch.empty_like(x) for _ in range(3))
        s = torch.cuda.current_stream(x.device).cuda_stream
        _lib.check("dn_density_forward", _lib.lib().dn_density_forward(
            ctypes.byref(d), x.data_ptr(), work.data_ptr(), filt.data_ptr(), eps.data_ptr(), s))
        ctx.save_for_backward(filt)
        ctx.d, ctx.shape = d, shape
        return eps.view(shape)

    @staticmethod
    def backward(ctx, g):
        (filt,) = ctx.saved_tensors
        gx = g.to(torch.float32).contiguous().view(filt.shape)
        work, drho = torch.empty_like(filt), torch.empty_like(filt)
        s = torch.cuda.current_stream(filt.device).cuda_stream
        _lib.check("dn_density_backward", _lib.lib().dn_density_backward(
            ctypes.byref(ctx.d), filt.data_ptr(), gx.data_ptr(), work.data_ptr(),
            drho.data_ptr(), s))
        return drho.view(ctx.shape), None, None, None, None, None, None


def density_to_eps(rho: torch.Tensor, radius: float = 2.0, beta: float = 1.0, eta: float = 0.5,
                   projection: str = "tanh", eps_lo: float = 1.0,
                   eps_hi: float = 12.1) -> torch.Tensor:
    """``eps = lo + (hi - lo) * project(smooth_filter(rho, radius))``, differentiable."""
    if projection not in KINDS:
        raise ValueError(f"projection must be one of {sorted(KINDS)}, got {projection!r}")
    return _DensityToEps.apply(rho, radius, beta, eta, projection, eps_lo, eps_hi)


def smooth_filter(density: torch.Tensor, radius: float = 2.0) -> torch.Tensor:
    return density_to_eps(density, radius, 1.0, 0.5, "none", 0.0, 1.0)


def heaviside_projection(density: torch.Tensor, beta: float = 10.0,
                         eta: float = 0.5) -> torch.Tensor:
    return density_to_eps(density, 0.0, beta, eta, "sigmoid", 0.0, 1.0)


def tanh_projection(density: torch.Tensor, beta: float = 10.0, eta: float = 0.5) -> torch.Tensor:
    return density_to_eps(density, 0.0, beta, eta, "tanh", 0.0, 1.0)


def beta_continuation_schedule(step: int, total_steps: int = 500, beta_start: float = 1.0,
                               beta_end: float = 64.0) -> float:
    t = min(step / total_steps, 1.0)
    return beta_start * (beta_end / beta_start) ** t


class _Morph3(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, dilate):
        shape = x.shape
        xl = _as_layers(x)
        L, H, W = xl.shape
        y = torch.empty_like(xl)
        arg = torch.empty(xl.shape, dtype=torch.int32, device=xl.device)
        s = torch.cuda.current_stream(xl.device).cuda_stream
        _lib.check("dn_morph3", _lib.lib().dn_morph3(xl.data_ptr(), L, H, W, int(dilate),
                                                     y.data_ptr(), arg.data_ptr(), s))
        ctx.save_for_backward(arg)
        ctx.shape = shape
        return y.view(shape)

    @staticmethod
    def backward(ctx, g):
        (arg,) = ctx.saved_tensors
        L, H, W = arg.shape
        gy = g.to(torch.float32).contiguous()
        dx = torch.empty(arg.shape, dtype=torch.float32, device=arg.device)
        s = torch.cuda.current_stream(arg.device).cuda_stream
        _lib.check("dn_morph3_backward", _lib.lib().dn_morph3_backward(
            gy.data_ptr(), arg.data_ptr(), L, H, W, dx.data_ptr(), s))
        return dx.view(ctx.shape), None


def erode(x: torch.Tensor) -> torch.Tensor:
    """One-cell erosion (3x3 min pool) in every layer, differentiable."""
    return _Morph3.apply(x, False)


def dilate(x: torch.Tensor) -> torch.Tensor:
    """One-cell dilation (3x3 max pool) in every layer, differentiable."""
    return _Morph3.apply(x, True)
