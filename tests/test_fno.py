"""Fourier-neural-operator surrogate: the DFT-matrix formulation against the
FFT oracle (CPU, FP64), and the GPU forward pass, every parameter gradient and
the input gradient against the oracle's FP32 autograd (GPU)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from diffnano_b200.surrogate.fno import (FNOConfig, dft_matrices, mode_table, padded_h_pass,
                                          separable_dft_matrices, t1_half)
from oracle import fno_ref

from conftest import rel_l2

# BF16 activations, BF16 DFT matrices and BF16 weight mirrors against an FP32
# FFT oracle fed the same BF16-rounded weights: a few BF16 roundings (2^-9)
# per layer, accumulated over 4 layers
TOL_FWD = 2e-2
TOL_GRAD = 5e-2


def test_dft_matrices_match_rfft2_irfft2():
    cfg = FNOConfig(H=32, W=24, width=8, modes=4)
    F2, G = dft_matrices(cfg)
    rng = np.random.default_rng(0)
    x = rng.standard_normal((2, 32, 24, 8))
    Z = np.einsum("mp,bpc->bmc", F2, x.reshape(2, 32 * 24, 8))
    kh, kw = mode_table(cfg)
    ref = np.fft.rfft2(x, axes=(1, 2))[:, kh, kw, :]
    assert np.abs(Z[:, :cfg.n_modes] - ref.real).max() < 1e-10
    assert np.abs(Z[:, cfg.n_modes:] - ref.imag).max() < 1e-10
    wre = torch.randn(cfg.n_modes, 8, 8, dtype=torch.float64)
    wim = torch.randn(cfg.n_modes, 8, 8, dtype=torch.float64)
    s = fno_ref.spectral(torch.from_numpy(x), wre, wim, 4).numpy()
    Yc = np.einsum("moi,bmi->bmo", (wre + 1j * wim).numpy(), ref)
    xs = np.einsum("pm,bmc->bpc", G, np.concatenate([Yc.real, Yc.imag], axis=1))
    assert np.abs(s - xs.reshape(s.shape)).max() < 1e-10


def _place(vals, out, row_radix, row0, row1, col_radix, col0, col1):
    """Store a (rows x cols) result through a GEMM output map (FP64 emulation)."""
    rows, cols = vals.shape
    r = np.arange(rows)[:, None]
    cc = np.arange(cols)[None, :]
    off = (r % row_radix) * row0 + (r // row_radix) * row1 \
        + (cc % col_radix) * col0 + (cc // col_radix) * col1
    out[off.reshape(-1)] = vals.reshape(-1)


@pytest.mark.parametrize("H,W,modes,B,C", [(32, 24, 4, 2, 8), (40, 64, 16, 1, 4),
                                           (10, 64, 4, 3, 4), (64, 32, 16, 2, 4)])
def test_separable_analysis_layout_matches_rfft2(H, W, modes, B, C):
    """The two transform passes of FNO2d._analysis, emulated in FP64 with the
    same output maps: the kept rfft2 modes land at dst[(m, re/im, b, c)]; the
    scaled W-pass matrix applies c_kw / (H W) per mode."""
    cfg = FNOConfig(H=H, W=W, width=C, modes=modes)
    Fw, FwS, Fh = separable_dft_matrices(cfg)
    M, R, NM = modes, B * C, cfg.n_modes
    Hp = t1_half(H)
    Fhp = padded_h_pass(Fh, H)
    rng = np.random.default_rng(1)
    x = rng.standard_normal((B, C, H, W))
    kh, kw = mode_table(cfg)
    ref = np.fft.rfft2(x, axes=(2, 3))[:, :, kh, kw]          # (B, C, NM)
    for F, scale in ((Fw, np.ones(NM)), (FwS, np.where(kw == 0, 1.0, 2.0) / (H * W))):
        T1 = np.zeros(M * R * 2 * Hp)
        if H % 32 == 0:  # the transposed first pass
            _place(F @ x.reshape(R * H, W).T, T1, M, R * 2 * Hp, Hp, H, 1, 2 * Hp)
        else:
            _place(x.reshape(R * H, W) @ F.T, T1, H, 1, 2 * Hp, M, R * 2 * Hp, Hp)
        dst = np.zeros(NM * 2 * R)
        _place(T1.reshape(M * R, 2 * Hp) @ Fhp.T, dst, R, 1, 2 * R, 2 * M, 2 * M * R, R)
        got = dst.reshape(NM, 2, B, C)
        want = ref.transpose(2, 0, 1) * scale[:, None, None]    # (NM, B, C)
        assert np.abs(got[:, 0] - want.real).max() < 1e-9
        assert np.abs(got[:, 1] - want.imag).max() < 1e-9


def _bf16_round(params):
    """The weights the GPU reads as BF16 GEMM operands, rounded the same way."""
    out = {}
    for k, v in params.items():
        if k in ("P", "Q1", "Q2") or k.startswith(("W", "wre", "wim")):
            v = v.to(torch.bfloat16).to(torch.float32)
        out[k] = v
    return out


def _design_batch(B, seed):
    from diffnano_b200.workloads import blob_eps_2d
    eps = torch.stack([blob_eps_2d(256, 128, seed=seed + i, sigma_cells=2 + i % 5)[64:192, 64:192]
                       for i in range(B)])
    return eps.to(torch.float32)


@pytest.mark.gpu
def test_fno_forward_and_gradients_match_oracle(cuda):
    from diffnano_b200.surrogate.fno import FNO2d
    cfg = FNOConfig()
    net = FNO2d(cfg, cuda, seed=3)
    params = _bf16_round({k: v for k, v in net.state_dict().items()})
    B = 4
    eps = _design_batch(B, 11)
    g = torch.Generator().manual_seed(5)
    target = torch.randn(B, cfg.W, cfg.n_out, generator=g) * 0.1
    kw = dict(layers=cfg.layers, modes=cfg.modes, n_out=cfg.n_out, lo=cfg.eps_lo, hi=cfg.eps_hi)
    loss_ref, pred_ref, grads_ref, deps_ref = fno_ref.loss_and_grads(params, eps, target, **kw)

    pred = net.forward(eps.to(cuda))
    loss = net.loss(target.to(cuda))
    net.ps.g.zero_()
    deps = net.backward(B=B, want_input_grad=True)
    torch.cuda.synchronize()
    net.check_status()
    assert rel_l2(pred, pred_ref) < TOL_FWD
    assert abs(float(loss) - float(loss_ref)) / float(loss_ref) < TOL_FWD
    for name, gref in grads_ref.items():
        gg = net.ps.G(name).cpu()
        if name == "P":
            gg, gref = gg[:, :3], gref[:, :3]
        if name in ("Q2", "q2"):
            gg, gref = gg[:cfg.n_out], gref[:cfg.n_out]
        err = rel_l2(gg, gref)
        assert err < TOL_GRAD, f"gradient of {name}: rel-L2 {err:.3e}"
    assert rel_l2(deps, deps_ref) < TOL_GRAD


@pytest.mark.gpu
def test_fno_adam_step_decreases_loss(cuda):
    from diffnano_b200.surrogate.fno import FNO2d
    cfg = FNOConfig()
    net = FNO2d(cfg, cuda, seed=4)
    B = 8
    eps = _design_batch(B, 21)
    # a learnable target: per-column fill fraction of the design, scaled per output
    fill = ((eps - cfg.eps_lo) / (cfg.eps_hi - cfg.eps_lo)).mean(dim=1)  # (B, W)
    scale = torch.linspace(-0.5, 0.5, cfg.n_out)
    target = (fill[:, :, None] - 0.5) * scale[None, None, :]
    eps, target = eps.to(cuda), target.to(cuda)
    losses = []
    for _ in range(30):
        net.forward(eps)
        losses.append(float(net.loss(target)))
        net.ps.g.zero_()
        net.backward(B=B)
        net.adam_step(lr=2e-3)
    torch.cuda.synchronize()
    net.check_status()
    assert losses[-1] < 0.5 * losses[0], losses


@pytest.mark.gpu
def test_fno_odd_batch_matches_even(cuda):
    """Samples are processed in pairs; an odd batch pads with a zero sample
    that must not leak into the real ones."""
    from diffnano_b200.surrogate.fno import FNO2d
    net = FNO2d(FNOConfig(), cuda, seed=7)
    eps = _design_batch(4, 31).to(cuda)
    full = net.forward(eps).clone()
    odd = net.forward(eps[:3]).clone()
    one = net.forward(eps[2:3]).clone()
    torch.cuda.synchronize()
    net.check_status()
    assert torch.equal(odd, full[:3])
    assert torch.equal(one[0], full[2])


@pytest.mark.gpu
@pytest.mark.parametrize("n_pix", [16384, 1003])
def test_lift_kernel_matches_lift_gemm(cuda, n_pix):
    """dn_fno_lift (the lifting layer as a memory-bound kernel) against the
    same contraction run as a K = 8 tensor-core GEMM with a row bias: equal up
    to one BF16 rounding step (the FP32 sums may be formed in another order);
    n_pix = 1003 takes the per-element store path."""
    from diffnano_b200 import _lib
    from diffnano_b200.surrogate.gemm import OutMap, gemm, kmajor

    nb, C, FEAT = 5, 64, 8
    g = torch.Generator().manual_seed(7)
    feat = torch.randn(nb, n_pix, FEAT, generator=g).to(torch.bfloat16).to(cuda)
    P = torch.randn(C, FEAT, generator=g).to(torch.bfloat16).to(cuda)
    bias = torch.randn(C, generator=g).to(cuda)
    x_kernel = torch.full((nb, C, n_pix), float("nan"), dtype=torch.bfloat16, device=cuda)
    x_gemm = torch.empty_like(x_kernel)
    s = torch.cuda.current_stream().cuda_stream
    _lib.check("dn_fno_lift", _lib.lib().dn_fno_lift(
        feat.data_ptr(), P.data_ptr(), bias.data_ptr(), nb, n_pix, C, x_kernel.data_ptr(), s))
    gemm(C, n_pix, [(kmajor(P, C, FEAT), kmajor(feat, n_pix, FEAT, batch_stride=n_pix * FEAT))],
         x_gemm, OutMap.rowmajor(n_pix, batch=C * n_pix), batch=nb, row_bias=bias)
    torch.cuda.synchronize()
    ref = torch.einsum("ck,bpk->bcp", P.double(), feat.double()) + bias.double()[None, :, None]
    mag = torch.einsum("ck,bpk->bcp", P.double().abs(), feat.double().abs()) \
        + bias.double().abs()[None, :, None]
    # half a BF16 step of the result (2^-8 relative) plus FP32 summation
    # error of 9 terms, with a margin
    bound = 1.01 * 2.0 ** -8 * ref.abs() + 2.0 ** -18 * mag
    for name, x in (("kernel", x_kernel), ("gemm", x_gemm)):
        d = (x.double() - ref).abs()
        assert bool((d <= bound).all()), (name, float((d / bound).max()))
    assert rel_l2(x_kernel.double(), x_gemm.double()) < 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("nm,nb,C", [(512, 4, 64), (130, 3, 70), (7, 2, 5)])
def test_modes_rows_permutation(cuda, nm, nb, C):
    """dn_fno_modes_rows both ways against torch's permute, bit for bit: the
    64 x 64 two-element kernel (even sizes, ragged tiles) and the 32 x 32 one
    (odd sizes)."""
    from diffnano_b200 import _lib

    g = torch.Generator().manual_seed(3)
    modes = torch.randn(nm, nb, 2, C, generator=g).to(torch.bfloat16).to(cuda)
    rows = torch.empty(nb, C, 2, nm, dtype=torch.bfloat16, device=cuda)
    back = torch.empty_like(modes)
    s = torch.cuda.current_stream().cuda_stream
    L = _lib.lib()
    _lib.check("dn_fno_modes_rows", L.dn_fno_modes_rows(
        modes.data_ptr(), rows.data_ptr(), nm, nb, C, 1, s))
    _lib.check("dn_fno_modes_rows", L.dn_fno_modes_rows(
        rows.data_ptr(), back.data_ptr(), nm, nb, C, 0, s))
    torch.cuda.synchronize()
    assert torch.equal(rows, modes.permute(1, 3, 2, 0))
    assert torch.equal(back, modes)


@pytest.mark.gpu
@pytest.mark.parametrize("rows,cols,bf16", [(32768, 6, True), (256, 4096, False), (1000, 37, False)])
def test_colsum_matches_torch(cuda, rows, cols, bf16):
    """dn_colsum (two-pass deterministic column sums) against an FP64 sum,
    overwrite and accumulate, and bit-identical on a repeat."""
    from diffnano_b200 import _lib

    L = _lib.lib()
    g = torch.Generator().manual_seed(11)
    x = torch.randn(rows, cols + 3, generator=g)
    x = x.to(torch.bfloat16) if bf16 else x
    x = x.to(cuda)
    n_scr = int(L.dn_colsum_scratch_elems(rows, cols))
    scratch = torch.empty(n_scr, device=cuda)
    out = torch.full((cols,), 5.0, device=cuda)
    s = torch.cuda.current_stream().cuda_stream
    dt = 2 if bf16 else 0

    def run(acc):
        _lib.check("dn_colsum", L.dn_colsum(x.data_ptr(), dt, rows, cols, cols + 3, out.data_ptr(),
                                            acc, scratch.data_ptr(), n_scr, s))

    run(0)
    first = out.clone()
    run(0)
    torch.cuda.synchronize()
    ref = x[:, :cols].double().sum(0)
    assert torch.equal(first, out)
    assert rel_l2(out.double(), ref) < 1e-6
    run(1)
    torch.cuda.synchronize()
    assert rel_l2(out.double(), 2 * ref) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("nm,co,ci", [(512, 64, 64), (9, 5, 7)])
def test_pack_modes_block_form(cuda, nm, co, ci):
    """dn_fno_pack_modes against [[wre, -wim], [wim, wre]] built by torch, bit
    for bit (even c_in: two entries per thread; odd: one)."""
    from diffnano_b200 import _lib

    g = torch.Generator().manual_seed(9)
    wre = torch.randn(nm, co, ci, generator=g).to(cuda)
    wim = torch.randn(nm, co, ci, generator=g).to(cuda)
    blk = torch.empty(nm, 2 * co, 2 * ci, dtype=torch.bfloat16, device=cuda)
    s = torch.cuda.current_stream().cuda_stream
    _lib.check("dn_fno_pack_modes", _lib.lib().dn_fno_pack_modes(
        wre.data_ptr(), wim.data_ptr(), nm, co, ci, blk.data_ptr(), s))
    torch.cuda.synchronize()
    ref = torch.cat([torch.cat([wre, -wim], 2), torch.cat([wim, wre], 2)], 1).to(torch.bfloat16)
    assert torch.equal(blk, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("nb,H,W,C", [(3, 128, 128, 64), (2, 9, 13, 5)])
def test_readout_matches_einsum(cuda, nb, H, W, C):
    """dn_fno_readout (four columns per thread when W % 4 == 0, else one)
    against an FP64 einsum of the same BF16 inputs, to one BF16 rounding."""
    from diffnano_b200 import _lib

    g = torch.Generator().manual_seed(13)
    x = torch.randn(nb, C, H, W, generator=g).to(torch.bfloat16).to(cuda)
    r = torch.randn(H, C, generator=g).to(cuda)
    out = torch.empty(nb, W, C, dtype=torch.bfloat16, device=cuda)
    s = torch.cuda.current_stream().cuda_stream
    _lib.check("dn_fno_readout", _lib.lib().dn_fno_readout(
        x.data_ptr(), r.data_ptr(), nb, H, W, C, out.data_ptr(), s))
    torch.cuda.synchronize()
    ref = torch.einsum("hc,bchw->bwc", r.double(), x.double())
    assert rel_l2(out.double(), ref) < 4e-3
