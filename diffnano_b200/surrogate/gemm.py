"""Python side of the BF16 tensor-core GEMM (``dn_gemm_run``, include/dn_fno.h).

Every contraction of the Fourier-neural-operator surrogate goes through
:func:`gemm`: ``C[z] = sum_s A_s[z] @ B_s[z]^T`` with BF16 operands, FP32
accumulation in tensor memory and a fused epilogue (scale, bias, addend, GELU
or its gradient) whose output index map lets one GEMM write the layout the
next one reads.  The operands and outputs are torch tensors on the current
CUDA device; the launch goes to the current stream.  There is no fallback:
without the CUDA library the call raises.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence, Tuple

import torch

from .. import _lib

DN_F32, DN_BF16 = 0, 2
ACT_NONE, ACT_GELU, ACT_GELU_GRAD = 0, 1, 2


@dataclass
class Operand:
    """A BF16 operand view: element (r, k) of batch z at
    K-major: ``z*batch_stride + r*ld + k``;
    MN-major: ``z*batch_stride + (r // fold)*fold_stride + k*ld + r % fold``
    (``fold = 0``: no fold), counted in elements from ``t``'s first element."""

    t: torch.Tensor
    rows: int
    k: int
    ld: int
    mn_major: bool = False
    fold: int = 0
    fold_stride: int = 0
    batch_stride: int = 0

    def c(self) -> _lib.DnGemmOperand:
        if self.t.dtype != torch.bfloat16 or not self.t.is_cuda:
            raise TypeError("GEMM operands are CUDA bfloat16 tensors")
        return _lib.DnGemmOperand(self.t.data_ptr(), int(self.mn_major), int(self.fold),
                                  int(self.rows), int(self.k), int(self.ld),
                                  int(self.fold_stride), int(self.batch_stride))


def kmajor(t: torch.Tensor, rows: int, k: int, ld: Optional[int] = None,
           batch_stride: int = 0) -> Operand:
    """Rows of ``k`` contiguous elements, ``ld`` apart (default ``k``)."""
    return Operand(t, rows, k, k if ld is None else ld, False, 0, 0, batch_stride)


def mnmajor(t: torch.Tensor, rows: int, k: int, ld: int, fold: int = 0, fold_stride: int = 0,
            batch_stride: int = 0) -> Operand:
    """Row index contiguous (in runs of ``fold``), contraction index ``ld`` apart."""
    return Operand(t, rows, k, ld, True, fold, fold_stride, batch_stride)


@dataclass
class OutMap:
    """``off(z, r, c) = z*batch + (r % row_radix)*row0 + (r // row_radix)*row1
    + (c % col_radix)*col0 + (c // col_radix)*col1`` (radix 0: no split)."""

    batch: int = 0
    row_radix: int = 0
    row0: int = 0
    row1: int = 0
    col_radix: int = 0
    col0: int = 1
    col1: int = 0

    @staticmethod
    def rowmajor(ld: int, batch: int = 0) -> "OutMap":
        return OutMap(batch=batch, row0=ld, col0=1)


def _dtype_code(t: Optional[torch.Tensor]) -> int:
    if t is None:
        return DN_F32
    if t.dtype == torch.float32:
        return DN_F32
    if t.dtype == torch.bfloat16:
        return DN_BF16
    raise TypeError(f"epilogue tensors are float32 or bfloat16, got {t.dtype}")


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    if t is None:
        return None
    if not t.is_cuda:
        raise TypeError("epilogue tensors live on the GPU")
    return t.data_ptr()


def gemm(M: int, N: int, segs: Sequence[Tuple[Operand, Operand]], out: torch.Tensor,
         omap: OutMap, *, batch: int = 1, accumulate: bool = False, alpha: float = 1.0,
         act: int = ACT_NONE, bias: Optional[torch.Tensor] = None,
         row_scale: Optional[torch.Tensor] = None, batch_scale: Optional[torch.Tensor] = None,
         col_scale: Optional[torch.Tensor] = None, row_bias: Optional[torch.Tensor] = None,
         addend: Optional[torch.Tensor] = None, aux: Optional[torch.Tensor] = None,
         pre: Optional[torch.Tensor] = None, block_n: int = 0, max_ctas: int = 0,
         pair: int = 0, status: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Launch one ``dn_gemm_run`` on the current stream; returns ``out``.
    ``pair``: 0 or 1 one-CTA tiles, 2 two-CTA 256 x 256 tiles (tcgen05
    cta_group::2; correct, but measured slower than one-CTA tiles on B200)."""
    if not 1 <= len(segs) <= 2:
        raise ValueError("one or two K segments")
    g = _lib.DnGemm()
    g.M, g.N, g.batch, g.n_seg = int(M), int(N), int(batch), len(segs)
    for i, (a, b) in enumerate(segs):
        g.a[i] = a.c()
        g.b[i] = b.c()
    for t in (bias, row_scale, batch_scale, col_scale, row_bias):
        if t is not None and (t.dtype != torch.float32 or not t.is_contiguous()):
            raise TypeError("bias / row_scale / batch_scale are contiguous float32")
    g.out = _ptr(out)
    g.out_dtype = _dtype_code(out)
    g.accumulate = int(accumulate)
    g.c_batch_stride, g.c_row_radix = omap.batch, omap.row_radix
    g.c_row_stride0, g.c_row_stride1 = omap.row0, omap.row1
    g.c_col_radix, g.c_col_stride0, g.c_col_stride1 = omap.col_radix, omap.col0, omap.col1
    g.alpha = float(alpha)
    g.act = int(act)
    g.bias, g.row_scale, g.batch_scale = _ptr(bias), _ptr(row_scale), _ptr(batch_scale)
    g.col_scale, g.row_bias = _ptr(col_scale), _ptr(row_bias)
    g.addend, g.addend_dtype = _ptr(addend), _dtype_code(addend)
    g.aux, g.aux_dtype = _ptr(aux), _dtype_code(aux)
    g.pre, g.pre_dtype = _ptr(pre), _dtype_code(pre)
    g.block_n, g.max_ctas, g.pair = int(block_n), int(max_ctas), int(pair)
    stream = torch.cuda.current_stream().cuda_stream
    st = None if status is None else status.data_ptr()
    _lib.check("dn_gemm_run", _lib.lib().dn_gemm_run(ctypes.byref(g), st, stream))
    return out
