"""Figure of merit sum |F|^2 of a monitor DFT, reduced in FP64 by the
``dn_fom_abs2`` kernel, differentiable (dFOM/dF = 2 F)."""

from __future__ import annotations

import ctypes

import torch

from diffnano_b200 import _lib


class _FomAbs2(torch.autograd.Function):
    @staticmethod
    def forward(ctx, f_real: torch.Tensor) -> torch.Tensor:
        f = f_real.contiguous()
        n = f.numel() // 2
        L = _lib.lib()
        nbytes = int(L.dn_fom_abs2_scratch_bytes(n))
        scratch = torch.empty((nbytes + 15) // 16 * 2, dtype=torch.float64, device=f.device)
        out = torch.empty((), dtype=torch.float64, device=f.device)
        with torch.cuda.device(f.device):
            stream = torch.cuda.current_stream(f.device).cuda_stream
            rc = L.dn_fom_abs2(f.data_ptr(), n, out.data_ptr(), scratch.data_ptr(),
                               scratch.numel() * 8, ctypes.c_void_p(stream))
        _lib.check("dn_fom_abs2", rc)
        ctx.save_for_backward(f)
        return out

    @staticmethod
    def backward(ctx, g):
        (f,) = ctx.saved_tensors
        return 2.0 * g * f


def fom_abs2(dft: torch.Tensor) -> torch.Tensor:
    """``sum |dft|^2`` (FP64 scalar) of a complex monitor DFT on a CUDA device."""
    if not dft.is_cuda:
        raise ValueError("fom_abs2 takes a CUDA tensor (the monitor DFTs of a solve)")
    z = dft.to(torch.complex128)
    return _FomAbs2.apply(torch.view_as_real(z.contiguous()).reshape(-1))
