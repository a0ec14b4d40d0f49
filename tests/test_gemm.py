"""The tcgen05 BF16 GEMM against a float64 torch product of the same BF16
inputs: operand layouts (K-major, MN-major, folded MN-major, shared and
batched), two K segments, K/M/N tails, every tile width, one-CTA and
two-CTA (256 x 256 pair) tiles, and the fused epilogue (scales, bias,
addend, GELU, GELU gradient, accumulate, BF16 output with 32- and 16-byte
aligned rows, index maps)."""

from __future__ import annotations

import ctypes

import pytest
import torch

from diffnano_b200 import _lib
from diffnano_b200.surrogate.gemm import (ACT_GELU, ACT_GELU_GRAD, OutMap, gemm, kmajor,
                                          mnmajor)

TOL_F32 = 2e-6  # FP32 accumulation of exact BF16 products (order differs)
TOL_BF16 = 8e-3  # one BF16 rounding of the result


def _rel(a, b) -> float:
    a, b = a.double().cpu(), b.double().cpu()
    return float((a - b).norm() / b.norm().clamp_min(1e-300))


def _bf(*shape, seed=0, dev="cuda"):
    g = torch.Generator().manual_seed(seed)
    return torch.randn(*shape, generator=g, dtype=torch.float32).to(torch.bfloat16).to(dev)


def _status(dev):
    return torch.zeros(1, dtype=torch.int32, device=dev)


def _check_status(st):
    assert int(st.item()) == 0, f"device status {int(st.item())}"


@pytest.mark.gpu
@pytest.mark.parametrize("block_n", [0, 64, 128, 256])
def test_kmajor_tails(cuda, block_n):
    M, N, K = 300, 200, 200
    a, b = _bf(M, K, seed=1), _bf(N, K, seed=2)
    out = torch.full((M, N), float("nan"), device=cuda)
    st = _status(cuda)
    gemm(M, N, [(kmajor(a, M, K), kmajor(b, N, K))], out, OutMap.rowmajor(N), block_n=block_n,
         status=st)
    torch.cuda.synchronize()
    _check_status(st)
    assert _rel(out, a.double() @ b.double().T) < TOL_F32


@pytest.mark.gpu
def test_tiny_and_persistent_loop(cuda):
    # one element; and more tiles than CTAs (each CTA walks several tiles and
    # both accumulator buffers)
    a, b = _bf(1, 8, seed=3), _bf(1, 8, seed=4)
    out = torch.zeros(1, 1, device=cuda)
    gemm(1, 1, [(kmajor(a, 1, 1, ld=8), kmajor(b, 1, 1, ld=8))], out, OutMap.rowmajor(1))
    torch.cuda.synchronize()
    assert abs(float(out) - float(a[0, 0].float() * b[0, 0].float())) < 1e-6
    M, N, K = 1024, 512, 192
    a, b = _bf(M, K, seed=5), _bf(N, K, seed=6)
    out = torch.zeros(M, N, device=cuda)
    st = _status(cuda)
    gemm(M, N, [(kmajor(a, M, K), kmajor(b, N, K))], out, OutMap.rowmajor(N), block_n=64,
         max_ctas=5, status=st)
    torch.cuda.synchronize()
    _check_status(st)
    assert _rel(out, a.double() @ b.double().T) < TOL_F32


@pytest.mark.gpu
@pytest.mark.parametrize("block_n", [64, 128, 256])
def test_mnmajor_operands(cuda, block_n):
    M, N, K = 256, 320, 130
    at = _bf(K, M, seed=7)  # A stored (K, M): M contiguous
    bt = _bf(K, N, seed=8)  # B stored (K, N)
    out = torch.zeros(M, N, device=cuda)
    st = _status(cuda)
    gemm(M, N, [(mnmajor(at, M, K, ld=M), mnmajor(bt, N, K, ld=N))], out, OutMap.rowmajor(N),
         block_n=block_n, status=st)
    torch.cuda.synchronize()
    _check_status(st)
    assert _rel(out, at.double().T @ bt.double()) < TOL_F32


@pytest.mark.gpu
def test_folded_mnmajor_b(cuda):
    # B[(b, c), hw] = X[b, hw, c]: channel-last activations read as one operand
    nb, HW, C, M = 5, 200, 64, 160
    x = _bf(nb, HW, C, seed=9)
    a = _bf(M, HW, seed=10)
    N = nb * C
    out = torch.zeros(M, N, device=cuda)
    b = mnmajor(x, N, HW, ld=C, fold=C, fold_stride=HW * C)
    gemm(M, N, [(kmajor(a, M, HW), b)], out, OutMap.rowmajor(N), block_n=256)
    torch.cuda.synchronize()
    B = x.double().permute(0, 2, 1).reshape(N, HW)
    assert _rel(out, a.double() @ B.T) < TOL_F32


@pytest.mark.gpu
def test_batched_shared_a_and_row_map(cuda):
    # A shared across 6 batches, B batched; C[z, r, c] written to
    # out[(r % 64), z, (r // 64), c] via a two-digit row map
    Z, M, N, K = 6, 128, 96, 64
    a = _bf(M, K, seed=11)
    b = _bf(Z, N, K, seed=12)
    out = torch.zeros(64, Z, 2, N, device=cuda)
    om = OutMap(batch=2 * N, row_radix=64, row0=Z * 2 * N, row1=N, col0=1)
    gemm(M, N, [(kmajor(a, M, K), kmajor(b, N, K, batch_stride=N * K))], out, om, batch=Z)
    torch.cuda.synchronize()
    ref = torch.einsum("mk,znk->zmn", a.double(), b.double())  # (Z, M, N)
    ref = ref.reshape(Z, 2, 64, N).permute(2, 0, 1, 3)
    assert _rel(out, ref) < TOL_F32


@pytest.mark.gpu
def test_two_segments_and_transposed_store(cuda):
    # C = A0 B0^T + A1 B1^T with segment 1 MN-major, stored transposed
    M, N, K0, K1 = 200, 64, 96, 64
    a0, b0 = _bf(M, K0, seed=13), _bf(N, K0, seed=14)
    a1t, b1 = _bf(K1, M, seed=15), _bf(N, K1, seed=16)
    out = torch.zeros(N, M, device=cuda)
    om = OutMap(row0=1, col0=M)
    gemm(M, N, [(kmajor(a0, M, K0), kmajor(b0, N, K0)),
                (mnmajor(a1t, M, K1, ld=M), kmajor(b1, N, K1))], out, om)
    torch.cuda.synchronize()
    ref = a0.double() @ b0.double().T + a1t.double().T @ b1.double().T
    assert _rel(out.T, ref) < TOL_F32


@pytest.mark.gpu
def test_epilogue_chain(cuda):
    Z, M, N, K = 3, 256, 128, 128
    a, b = _bf(Z, M, K, seed=17), _bf(N, K, seed=18)
    g = torch.Generator().manual_seed(19)
    bias = torch.randn(N, generator=g).to(cuda)
    rs = (torch.rand(M, generator=g) + 0.5).to(cuda)
    bs = (torch.rand(Z, generator=g) + 0.5).to(cuda)
    addend = torch.randn(Z, M, N, generator=g).to(torch.bfloat16).to(cuda)
    acc = torch.einsum("zmk,nk->zmn", a.double(), b.double())
    v = 0.5 * acc * rs.double()[None, :, None] * bs.double()[:, None, None] + bias.double() \
        + addend.double()
    ops = [(kmajor(a, M, K, batch_stride=M * K), kmajor(b, N, K))]
    om = OutMap.rowmajor(N, batch=M * N)
    y = torch.zeros(Z, M, N, dtype=torch.bfloat16, device=cuda)
    pre = torch.zeros(Z, M, N, dtype=torch.bfloat16, device=cuda)
    gemm(M, N, ops, y, om, batch=Z, alpha=0.5, act=ACT_GELU, bias=bias, row_scale=rs,
         batch_scale=bs, addend=addend, pre=pre)
    torch.cuda.synchronize()
    assert _rel(pre, v) < TOL_BF16
    assert _rel(y, torch.nn.functional.gelu(v, approximate="tanh")) < TOL_BF16
    # gradient form, accumulated onto an FP32 output
    base = torch.randn(Z, M, N, generator=g).to(cuda)
    out = base.clone()
    gemm(M, N, ops, out, om, batch=Z, act=ACT_GELU_GRAD, aux=pre, accumulate=True)
    torch.cuda.synchronize()
    x = pre.double().requires_grad_(True)
    gp, = torch.autograd.grad(torch.nn.functional.gelu(x, approximate="tanh").sum(), x)
    assert _rel(out, base.double() + acc * gp) < 1e-5


@pytest.mark.gpu
def test_scalar_epilogue_path(cuda):
    # column stride != 1 and N not a multiple of 32: per-element stores
    M, N, K = 130, 45, 72
    a, b = _bf(M, K, seed=20), _bf(N, K, seed=21)
    out = torch.zeros(N, 3, M, device=cuda)
    om = OutMap(row0=1, col0=3 * M)
    gemm(M, N, [(kmajor(a, M, K), kmajor(b, N, K))], out, om)
    torch.cuda.synchronize()
    assert _rel(out[:, 0, :].T, a.double() @ b.double().T) < TOL_F32
    assert float(out[:, 1:, :].abs().max()) == 0.0


@pytest.mark.gpu
def test_bf16_rows_16_byte_aligned(cuda):
    # BF16 output rows 272 bytes apart: 16-byte but not 32-byte aligned, so
    # the epilogue takes its 16-byte store path
    M, N, K, LD = 200, 128, 96, 136
    a, b = _bf(M, K, seed=42), _bf(N, K, seed=43)
    out = torch.zeros(M, LD, dtype=torch.bfloat16, device=cuda)
    st = _status(cuda)
    gemm(M, N, [(kmajor(a, M, K), kmajor(b, N, K))], out, OutMap.rowmajor(LD), status=st)
    torch.cuda.synchronize()
    _check_status(st)
    assert _rel(out[:, :N], a.double() @ b.double().T) < TOL_BF16
    assert float(out[:, N:].abs().max()) == 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,K,max_ctas", [
    (300, 200, 200, 0),    # ragged pair tile: the second CTA's rows partly past M
    (100, 256, 64, 0),     # the second CTA's rows entirely past M
    (130, 520, 1000, 0),   # N tail inside the second half of B; long K
    (1100, 700, 576, 4),   # two pairs walk many tiles: both accumulator buffers, ring wraps
])
def test_pair_tiles_kmajor(cuda, M, N, K, max_ctas):
    a, b = _bf(M, K, seed=31), _bf(N, K, seed=32)
    ref = a.double() @ b.double().T
    for pair in (1, 2):
        out = torch.full((M, N), float("nan"), device=cuda)
        st = _status(cuda)
        gemm(M, N, [(kmajor(a, M, K), kmajor(b, N, K))], out, OutMap.rowmajor(N), pair=pair,
             max_ctas=max_ctas, status=st)
        torch.cuda.synchronize()
        _check_status(st)
        assert _rel(out, ref) < TOL_F32, f"pair={pair}"


@pytest.mark.gpu
def test_pair_tiles_mnmajor_and_fold(cuda):
    M, N, K = 384, 640, 130
    at, bt = _bf(K, M, seed=33), _bf(K, N, seed=34)
    out = torch.zeros(M, N, device=cuda)
    st = _status(cuda)
    gemm(M, N, [(mnmajor(at, M, K, ld=M), mnmajor(bt, N, K, ld=N))], out, OutMap.rowmajor(N),
         pair=2, status=st)
    torch.cuda.synchronize()
    _check_status(st)
    assert _rel(out, at.double().T @ bt.double()) < TOL_F32
    # B[(b, c), hw] = X[b, hw, c] folded by C = 64 channels
    nb, HW, C, M2 = 7, 200, 64, 300
    x, a = _bf(nb, HW, C, seed=35), _bf(M2, HW, seed=36)
    N2 = nb * C
    out = torch.zeros(M2, N2, device=cuda)
    gemm(M2, N2, [(kmajor(a, M2, HW), mnmajor(x, N2, HW, ld=C, fold=C, fold_stride=HW * C))],
         out, OutMap.rowmajor(N2), pair=2, status=st)
    torch.cuda.synchronize()
    _check_status(st)
    B = x.double().permute(0, 2, 1).reshape(N2, HW)
    assert _rel(out, a.double() @ B.T) < TOL_F32


@pytest.mark.gpu
def test_pair_tiles_segments_batch_epilogue(cuda):
    # two K segments (K-major A0, MN-major A1), batched A and shared B, the
    # full epilogue into BF16 with a transposed store
    Z, M, N, K0, K1 = 3, 320, 288, 192, 64
    a0, b0 = _bf(Z, M, K0, seed=37), _bf(N, K0, seed=38)
    a1t, b1 = _bf(Z, K1, M, seed=39), _bf(N, K1, seed=40)
    g = torch.Generator().manual_seed(41)
    bias = torch.randn(N, generator=g).to(cuda)
    rb = torch.randn(M, generator=g).to(cuda)
    cs = (torch.rand(N, generator=g) + 0.5).to(cuda)
    bs = (torch.rand(Z, generator=g) + 0.5).to(cuda)
    acc = torch.einsum("zmk,nk->zmn", a0.double(), b0.double()) \
        + torch.einsum("zkm,nk->zmn", a1t.double(), b1.double())
    v = acc * cs.double() * bs.double()[:, None, None] + bias.double() + rb.double()[:, None]
    y = torch.zeros(Z, N, M, dtype=torch.bfloat16, device=cuda)
    om = OutMap(batch=N * M, row0=1, col0=M)
    st = _status(cuda)
    gemm(M, N, [(kmajor(a0, M, K0, batch_stride=M * K0), kmajor(b0, N, K0)),
                (mnmajor(a1t, M, K1, ld=M, batch_stride=K1 * M), kmajor(b1, N, K1))],
         y, om, batch=Z, act=ACT_GELU, bias=bias, row_bias=rb, col_scale=cs, batch_scale=bs,
         pair=2, status=st)
    torch.cuda.synchronize()
    _check_status(st)
    assert _rel(y.transpose(1, 2), torch.nn.functional.gelu(v, approximate="tanh")) < TOL_BF16


def test_gemm_rejects_bad_arguments():
    """Host-side validation (no GPU work): misaligned strides and mismatched K."""
    L = _lib.lib()
    g = _lib.DnGemm()
    g.M, g.N, g.batch, g.n_seg = 16, 16, 1, 1
    fake = 1 << 20  # 16-byte aligned, never dereferenced: validation fails first
    g.a[0] = _lib.DnGemmOperand(fake, 0, 0, 16, 16, 7, 0, 0)  # ld not a multiple of 8
    g.b[0] = _lib.DnGemmOperand(fake, 0, 0, 16, 16, 16, 0, 0)
    g.out = fake
    assert L.dn_gemm_run(ctypes.byref(g), None, None) == 1
    g.a[0] = _lib.DnGemmOperand(fake, 0, 0, 16, 24, 24, 0, 0)  # K 24 vs 16
    assert L.dn_gemm_run(ctypes.byref(g), None, None) == 1
    g.a[0] = _lib.DnGemmOperand(fake, 1, 32, 16, 16, 16, 64, 0)  # fold not a multiple of 64
    assert L.dn_gemm_run(ctypes.byref(g), None, None) == 1
    g.a[0] = _lib.DnGemmOperand(fake, 0, 0, 16, 16, 16, 0, 0)
    g.block_n = 96
    assert L.dn_gemm_run(ctypes.byref(g), None, None) == 1
    g.block_n = 0
    g.accumulate, g.out_dtype = 1, 2  # accumulate into BF16
    assert L.dn_gemm_run(ctypes.byref(g), None, None) == 1
    g.accumulate, g.out_dtype = 0, 0
    g.pair = 3  # not a tile mode
    assert L.dn_gemm_run(ctypes.byref(g), None, None) == 1
    g.pair, g.block_n = 2, 64  # pair tiles are 256 wide
    assert L.dn_gemm_run(ctypes.byref(g), None, None) == 1
