"""Fourier neural operator (2-D) whose every contraction runs on the project's
BF16 tcgen05 GEMM (``dn_gemm_run``), forward and backward, with FP32
accumulation and FP32 master weights trained by the ``dn_adam`` kernel.

Network (channel-last activations ``X[b, h, w, c]``, BF16):

* features ``f = ((eps - lo) / (hi - lo), x, y)`` (8 slots), lifted to
  ``width`` channels: ``X0 = f P^T + p``;
* ``layers`` Fourier layers ``X_{l+1} = act(S_l(X_l) + X_l W_l^T + b_l)`` (GELU
  on all but the last), where ``S_l`` keeps ``modes`` x ``modes`` complex
  Fourier modes (rows ``kh`` in ``0..modes-1`` and ``H-modes..H-1``, columns
  ``kw`` in ``0..modes-1``, the rfft2 half-plane), mixes channels per mode
  with complex weights and transforms back (irfft2);
* readout: a learned weighted sum over rows ``R[b, w, c] = sum_h r[h, c]
  X[b, h, w, c]``, then ``GELU(R Q1^T + q1) Q2^T + q2`` -> ``n_out`` values per
  column (the monitor line: re/im of the DFT field at each wavelength).

The truncated 2-D DFT and its inverse are dense GEMMs against BF16 DFT
matrices (``F2``: 2*modes^2*2 x H*W, ``G = F2^T diag(c/HW)``), so one GEMM
transforms a whole batch with the modes on the tensor cores; the per-mode
complex mixing is a batched real GEMM over the 2x2 block form
``[[Wre, -Wim], [Wim, Wre]]``; the inverse transform and the 1x1 channel mix
share one GEMM (two K segments) whose epilogue adds the bias, applies GELU and
keeps the pre-activation for the backward pass.  Each GEMM's output index map
writes the layout the next GEMM reads, so no transposes run between them.

The oracle for this module is a torch FP32 CPU restatement with
``torch.fft.rfft2`` / ``irfft2`` and autograd (``oracle/fno_ref.py``).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from typing import Dict, Optional, Tuple

import numpy as np
import torch

from .. import _lib
from .gemm import ACT_GELU, ACT_GELU_GRAD, OutMap, gemm, kmajor, mnmajor

FEAT = 8  # feature slots per pixel (3 used)
OUT_LD = 8  # padded output columns per monitor point


@dataclass(frozen=True)
class FNOConfig:
    H: int = 128
    W: int = 128
    width: int = 64
    modes: int = 16
    layers: int = 4
    hidden: int = 128
    n_out: int = 6  # re/im at 3 wavelengths
    eps_lo: float = 2.085
    eps_hi: float = 12.1

    @property
    def n_modes(self) -> int:
        return 2 * self.modes * self.modes  # complex modes kept

    @property
    def n_mode_rows(self) -> int:
        return 2 * self.n_modes  # real rows of F2 (cos block, sin block)


def mode_table(cfg: FNOConfig) -> Tuple[np.ndarray, np.ndarray]:
    """(kh, kw) of every kept mode, index m = khi * modes + kw, khi < 2*modes."""
    khi = np.arange(2 * cfg.modes)
    kh = np.where(khi < cfg.modes, khi, khi - 2 * cfg.modes + cfg.H)
    kw = np.arange(cfg.modes)
    KH, KW = np.meshgrid(kh, kw, indexing="ij")
    return KH.reshape(-1), KW.reshape(-1)


def dft_matrices(cfg: FNOConfig) -> Tuple[np.ndarray, np.ndarray]:
    """F2 (2*n_modes, H*W) and G (H*W, 2*n_modes) in float64.

    F2[m, hw] = cos(theta), F2[n_modes + m, hw] = -sin(theta), theta =
    2*pi*(kh*h/H + kw*w/W): the rfft2 coefficients Re, Im of the kept modes.
    G = F2^T * c_kw / (H*W), c = 1 for kw = 0 else 2: the irfft2 synthesis
    from those modes (the imaginary part of the kw = 0 column drops out as in
    irfft2)."""
    kh, kw = mode_table(cfg)
    h = np.arange(cfg.H)
    w = np.arange(cfg.W)
    th = 2 * np.pi * (np.outer(kh, h)[:, :, None] / cfg.H + np.outer(kw, w)[:, None, :] / cfg.W)
    th = th.reshape(cfg.n_modes, cfg.H * cfg.W)
    F2 = np.concatenate([np.cos(th), -np.sin(th)], axis=0)
    c = np.where(kw == 0, 1.0, 2.0) / (cfg.H * cfg.W)
    G = (F2 * np.concatenate([c, c])[:, None]).T
    return F2, G


def separable_dft_matrices(cfg: FNOConfig) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """The truncated rfft2 of dft_matrices as a pass along W then one along H,
    in float64:

    Fw (2*modes, W): Fw[ri*modes + kw, w] = cos / -sin(2 pi kw w / W), so the
    W pass gives T = sum_w x e^{-i th_w} as (Re, Im) pairs;
    FwS: Fw with row (ri, kw) scaled by c_kw / (H W) (c = 1 for kw = 0, else 2),
    the analysis of the adjoint of the synthesis G;
    Fh (4*modes, 2*H): Z = sum_h T e^{-i th_h} as a real map from (Re T, Im T)
    over h to (Re Z, Im Z) over khi: [[cos, sin], [-sin, cos]] of
    th_h = 2 pi kh h / H, kh as in mode_table."""
    M = cfg.modes
    kw = np.arange(M)
    tw = 2 * np.pi * np.outer(kw, np.arange(cfg.W)) / cfg.W
    Fw = np.concatenate([np.cos(tw), -np.sin(tw)], axis=0)
    c = np.where(kw == 0, 1.0, 2.0) / (cfg.H * cfg.W)
    FwS = Fw * np.concatenate([c, c])[:, None]
    khi = np.arange(2 * M)
    kh = np.where(khi < M, khi, khi - 2 * M + cfg.H)
    th = 2 * np.pi * np.outer(kh, np.arange(cfg.H)) / cfg.H
    Ch, Sh = np.cos(th), np.sin(th)
    Fh = np.block([[Ch, Sh], [-Sh, Ch]])
    return Fw, FwS, Fh


def t1_half(H: int) -> int:
    """Length of each (Re, Im) half of a T1 row: H rounded up to a multiple of
    4, so that rows of 2 * t1_half(H) elements are valid GEMM operands."""
    return (H + 3) // 4 * 4


def padded_h_pass(Fh: np.ndarray, H: int) -> np.ndarray:
    """Fh (4*modes, 2*H) with each half of its columns zero-padded to t1_half(H)."""
    Hp = t1_half(H)
    out = np.zeros((Fh.shape[0], 2 * Hp))
    out[:, :H] = Fh[:, :H]
    out[:, Hp:Hp + H] = Fh[:, H:]
    return out


class ParamSet:
    """FP32 master parameters in one flat buffer (each tensor 8-element
    aligned so that its BF16 mirror is a valid GEMM operand), with the
    gradient buffer, Adam moments and the BF16 mirror in the same layout."""

    def __init__(self, shapes: Dict[str, Tuple[int, ...]], device: torch.device):
        self.offsets: Dict[str, Tuple[int, Tuple[int, ...]]] = {}
        off = 0
        for name, shp in shapes.items():
            self.offsets[name] = (off, shp)
            off += (int(np.prod(shp)) + 7) // 8 * 8
        self.n = off
        self.p = torch.zeros(off, device=device)
        self.g = torch.zeros(off, device=device)
        self.m = torch.zeros(off, device=device)
        self.v = torch.zeros(off, device=device)
        self.bf = torch.zeros(off, dtype=torch.bfloat16, device=device)
        self.step = 0

    def view(self, buf: torch.Tensor, name: str) -> torch.Tensor:
        off, shp = self.offsets[name]
        return buf[off:off + int(np.prod(shp))].view(shp)

    def P(self, name):  # noqa: N802 - parameter view
        return self.view(self.p, name)

    def G(self, name):  # noqa: N802 - gradient view
        return self.view(self.g, name)

    def B(self, name):  # noqa: N802 - BF16 mirror view
        return self.view(self.bf, name)


def _c(x) -> Optional[int]:
    return None if x is None else x.data_ptr()


class FNO2d:
    """The operator with its forward, backward and Adam step on one GPU."""

    def __init__(self, cfg: FNOConfig = FNOConfig(), device=None, seed: int = 0):
        self.cfg = cfg
        self.dev = torch.device(device) if device is not None else torch.device("cuda")
        if self.dev.type != "cuda":
            raise ValueError("FNO2d runs on a CUDA device")
        self.L = _lib.lib()
        c = cfg
        shapes: Dict[str, Tuple[int, ...]] = {"P": (c.width, FEAT), "p": (c.width,)}
        for l in range(c.layers):
            shapes[f"wre{l}"] = (c.n_modes, c.width, c.width)
            shapes[f"wim{l}"] = (c.n_modes, c.width, c.width)
            shapes[f"W{l}"] = (c.width, c.width)
            shapes[f"b{l}"] = (c.width,)
        shapes.update({"r": (c.H, c.width), "Q1": (c.hidden, c.width), "q1": (c.hidden,),
                       "Q2": (OUT_LD, c.hidden), "q2": (OUT_LD,)})
        self.ps = ParamSet(shapes, self.dev)
        self._init_params(seed)
        if 32 % c.modes and c.modes % 32:
            raise ValueError("modes must divide 32 or be a multiple of 32 (the transform "
                             "passes' output maps)")
        _, G = dft_matrices(c)
        self.Gm = torch.from_numpy(G).to(torch.bfloat16).to(self.dev).contiguous()
        Fw, FwS, Fh = separable_dft_matrices(c)
        bfd = dict(dtype=torch.bfloat16, device=self.dev)
        self.Fw = torch.from_numpy(Fw).to(**bfd).contiguous()
        self.FwS = torch.from_numpy(FwS).to(**bfd).contiguous()
        self.Fh = torch.from_numpy(padded_h_pass(Fh, c.H)).to(**bfd).contiguous()
        self.blk = [torch.empty(c.n_modes, 2 * c.width, 2 * c.width, dtype=torch.bfloat16,
                                device=self.dev) for _ in range(c.layers)]
        # 1x1 mixes of a sample pair: blockdiag(W, W), blockdiag(W^T, W^T), [b, b]
        pw = dict(dtype=torch.bfloat16, device=self.dev)
        self.pw = [torch.empty(2 * c.width, 2 * c.width, **pw) for _ in range(c.layers)]
        self.pwT = [torch.empty(2 * c.width, 2 * c.width, **pw) for _ in range(c.layers)]
        self.pw_bias = [torch.empty(2 * c.width, device=self.dev) for _ in range(c.layers)]
        # cw = c_kw / (H W) per mode (c = 1 for kw = 0, else 2); the mixing
        # backward's HW/c per mode turns the synthesis G into the analysis F2^T
        _, kw = mode_table(c)
        cw = torch.from_numpy(np.where(kw == 0, 1.0, 2.0) / (c.H * c.W)).to(torch.float32)
        self.bscale = (1.0 / cw).to(self.dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self._ws: Dict[int, Dict[str, torch.Tensor]] = {}
        self.refresh()

    # ---- parameters -------------------------------------------------------
    def _init_params(self, seed: int) -> None:
        c, ps = self.cfg, self.ps
        g = torch.Generator().manual_seed(seed)

        def unif(shape, bound):
            return (torch.rand(shape, generator=g, dtype=torch.float64) * 2 - 1) * bound

        P = torch.zeros(c.width, FEAT, dtype=torch.float64)
        P[:, :3] = unif((c.width, 3), 1 / math.sqrt(3))
        vals = {"P": P, "p": unif((c.width,), 1 / math.sqrt(3))}
        scale = 1.0 / (c.width * c.width)
        for l in range(c.layers):
            vals[f"wre{l}"] = scale * torch.rand((c.n_modes, c.width, c.width), generator=g,
                                                 dtype=torch.float64)
            vals[f"wim{l}"] = scale * torch.rand((c.n_modes, c.width, c.width), generator=g,
                                                 dtype=torch.float64)
            vals[f"W{l}"] = unif((c.width, c.width), 1 / math.sqrt(c.width))
            vals[f"b{l}"] = unif((c.width,), 1 / math.sqrt(c.width))
        vals["r"] = torch.full((c.H, c.width), 1.0 / c.H, dtype=torch.float64) \
            + unif((c.H, c.width), 0.1 / c.H)
        vals["Q1"] = unif((c.hidden, c.width), 1 / math.sqrt(c.width))
        vals["q1"] = unif((c.hidden,), 1 / math.sqrt(c.width))
        Q2 = torch.zeros(OUT_LD, c.hidden, dtype=torch.float64)
        Q2[:c.n_out] = unif((c.n_out, c.hidden), 1 / math.sqrt(c.hidden))
        vals["Q2"] = Q2
        vals["q2"] = torch.zeros(OUT_LD, dtype=torch.float64)
        for k, v in vals.items():
            ps.P(k).copy_(v.to(torch.float32))

    def state_dict(self) -> Dict[str, torch.Tensor]:
        """FP32 parameters by name (CPU copies)."""
        return {k: self.ps.P(k).detach().cpu().clone() for k in self.ps.offsets}

    def load_state_dict(self, sd: Dict[str, torch.Tensor]) -> None:
        for k, v in sd.items():
            self.ps.P(k).copy_(v.to(self.dev, torch.float32))
        self.refresh()

    def refresh(self) -> None:
        """Rebuild the BF16 operands from the FP32 masters."""
        L, c, s = self.L, self.cfg, self._stream()
        _lib.check("dn_f32_to_bf16", L.dn_f32_to_bf16(_c(self.ps.p), self.ps.n, _c(self.ps.bf), s))
        self._pack()

    def _pack(self) -> None:
        L, c, s = self.L, self.cfg, self._stream()
        for l in range(c.layers):
            _lib.check("dn_fno_pack_modes", L.dn_fno_pack_modes(
                _c(self.ps.P(f"wre{l}")), _c(self.ps.P(f"wim{l}")), c.n_modes, c.width,
                c.width, _c(self.blk[l]), s))
            _lib.check("dn_fno_pack_pointwise", L.dn_fno_pack_pointwise(
                _c(self.ps.P(f"W{l}")), _c(self.ps.P(f"b{l}")), c.width, _c(self.pw[l]),
                _c(self.pwT[l]), _c(self.pw_bias[l]), s))

    @staticmethod
    def _stream() -> int:
        return torch.cuda.current_stream().cuda_stream

    # ---- workspace ----------------------------------------------------------
    def _workspace(self, B: int) -> Dict[str, torch.Tensor]:
        if B in self._ws:
            return self._ws[B]
        c, d = self.cfg, self.dev
        HW, C, NM, NR = c.H * c.W, c.width, c.n_modes, c.n_mode_rows
        Bp = B + (B & 1)  # pair tensors: an even number of samples, the spare one zero
        bf = dict(dtype=torch.bfloat16, device=d)
        ws = {
            "feat": torch.zeros(B, HW, FEAT, **bf),
            "X": [torch.zeros(Bp, C, HW, **bf) for _ in range(c.layers + 1)],
            "pre": [torch.zeros(Bp, C, HW, **bf) for _ in range(c.layers - 1)],
            # kept modes of each layer's input, (mode, re/im, sample, channel)
            "Zm": [torch.empty(NM, 2, B, C, **bf) for _ in range(c.layers)],
            # W-pass output of the transform, ((kw, sample, channel), (re/im, h)),
            # each half padded to t1_half(H); zeroed once, the pad stays zero
            "T1": torch.zeros(c.modes * B * C, 2 * t1_half(c.H), **bf),
            "Ym": torch.empty(NM, B, 2 * C, **bf),
            "Yt": torch.zeros(Bp, C, NR, **bf),
            "R": torch.empty(B, c.W, C, **bf),
            "U": torch.empty(B * c.W, c.hidden, **bf),
            "preU": torch.empty(B * c.W, c.hidden, **bf),
            "out": torch.empty(B * c.W, OUT_LD, dtype=torch.float32, device=d),
        }
        self._ws[B] = ws
        return ws

    def _bwd_workspace(self, B: int) -> Dict[str, torch.Tensor]:
        ws = self._workspace(B)
        if "gout" in ws:
            return ws
        c, d = self.cfg, self.dev
        HW, C, NM, NR = c.H * c.W, c.width, c.n_modes, c.n_mode_rows
        Bp = B + (B & 1)
        bf = dict(dtype=torch.bfloat16, device=d)
        f32 = dict(dtype=torch.float32, device=d)
        ws.update({
            "gout": torch.zeros(B * c.W, OUT_LD, **bf),
            "dpreU": torch.empty(B * c.W, c.hidden, **bf),
            "dR": torch.empty(B * c.W, C, **bf),
            "dA": torch.zeros(Bp, C, HW, **bf),
            "dB": torch.zeros(Bp, C, HW, **bf),
            "dYm": torch.empty(NM, 2, B, C, **bf),
            "dZm": torch.empty(NM, B, 2 * C, **bf),
            "dZt": torch.zeros(Bp, C, NR, **bf),
            "dblk": torch.empty(NM, 2 * C, 2 * C, **f32),
            "part": torch.empty(B * max(c.H, c.hidden, OUT_LD) * max(C, c.hidden), **f32),
            "scratch": torch.empty(int(self.L.dn_colsum_scratch_elems(max(B * c.W, B),
                                                                       4 * C * C)), **f32),
            "loss_part": torch.zeros(256, dtype=torch.float64, device=d),
        })
        return ws

    def _analysis(self, src, Fw, dst, ws, B):
        """dst (modes, re/im, B, C) = the kept rfft2 modes of every (sample,
        channel) image of src (B, C, H, W) channel-first, in two GEMMs: along W
        (K = W, rows (sample, channel, h), into T1 ordered ((kw, sample,
        channel), (re/im, h))), then along H (K = 2H, rows (kw, sample,
        channel), columns (re/im, khi)), written straight into the
        per-mode layout.  Fw: self.Fw, or self.FwS for the adjoint of the
        synthesis.  ~30x fewer FLOPs than one dense (2 n_modes x H W) GEMM."""
        c, st = self.cfg, self.status
        M, H, W, R = c.modes, c.H, c.W, B * c.width
        Hp = t1_half(H)
        T1 = ws["T1"]
        if H % 32 == 0:
            # as T1^T = Fw X^T: rows (re/im, kw), columns (sample, channel, h)
            # with h contiguous in T1, so the epilogue stores whole 32-column runs
            gemm(2 * M, R * H, [(kmajor(Fw, 2 * M, W), kmajor(src, R * H, W))], T1,
                 OutMap(row_radix=M, row0=R * 2 * Hp, row1=Hp, col_radix=H, col0=1,
                        col1=2 * Hp), status=st)
        else:
            gemm(R * H, 2 * M, [(kmajor(src, R * H, W), kmajor(Fw, 2 * M, W))], T1,
                 OutMap(row_radix=H, row0=1, row1=2 * Hp, col_radix=M, col0=R * 2 * Hp,
                        col1=Hp), status=st)
        gemm(M * R, 4 * M, [(kmajor(T1, M * R, 2 * Hp), kmajor(self.Fh, 4 * M, 2 * Hp))], dst,
             OutMap(row_radix=R, row0=1, row1=2 * R, col_radix=2 * M, col0=2 * M * R, col1=R),
             status=st)

    def _modes_rows(self, src, dst, B, to_rows):
        c = self.cfg
        _lib.check("dn_fno_modes_rows", self.L.dn_fno_modes_rows(
            _c(src), _c(dst), c.n_modes, B, c.width, int(to_rows), self._stream()))

    # ---- passes -----------------------------------------------------------
    def forward(self, eps: torch.Tensor) -> torch.Tensor:
        """eps (B, H, W) float32 on the device -> prediction (B, W, n_out) float32."""
        c = self.cfg
        if eps.dim() != 3 or eps.shape[1:] != (c.H, c.W):
            raise ValueError(f"eps must be (B, {c.H}, {c.W}), got {tuple(eps.shape)}")
        eps = eps.to(self.dev, torch.float32).contiguous()
        B = eps.shape[0]
        ws = self._workspace(B)
        self._forward(eps, ws, B)
        return ws["out"].view(B, c.W, OUT_LD)[:, :, :c.n_out]

    def _forward(self, eps, ws, B):
        c, ps, L, s = self.cfg, self.ps, self.L, self._stream()
        HW, C, NM, NR = c.H * c.W, c.width, c.n_modes, c.n_mode_rows
        Bp = B + (B & 1)
        st = self.status
        _lib.check("dn_fno_features", L.dn_fno_features(
            _c(eps), B, c.H, c.W, c.eps_lo, c.eps_hi, _c(ws["feat"]), s))
        X = ws["X"]
        # lift, per sample X0[c, hw] = P feat^T + p (channel-first rows): a
        # K = 8 contraction, so a memory-bound kernel rather than a GEMM
        _lib.check("dn_fno_lift", L.dn_fno_lift(
            _c(ws["feat"]), _c(ps.B("P")), _c(ps.P("p")), B, HW, C, _c(X[0]), s))
        for l in range(c.layers):
            # truncated DFT of every (sample, channel) image: Zm[m, ri, b, c]
            Zl = ws["Zm"][l]
            self._analysis(X[l], self.Fw, Zl, ws, B)
            # per-mode complex channel mixing: Ym[m, b, (ri, o)]; K = (ri, c) as
            # two segments (the re and im halves of Zm and of blk's columns)
            blk = self.blk[l]
            gemm(B, 2 * C, [(kmajor(Zl, B, C, batch_stride=2 * B * C),
                             kmajor(blk, 2 * C, C, ld=2 * C, batch_stride=4 * C * C)),
                            (kmajor(Zl.view(-1)[B * C:], B, C, batch_stride=2 * B * C),
                             kmajor(blk.view(-1)[C:], 2 * C, C, ld=2 * C,
                                    batch_stride=4 * C * C))],
                 ws["Ym"], OutMap.rowmajor(2 * C, batch=B * 2 * C), batch=NM, status=st)
            self._modes_rows(ws["Ym"], ws["Yt"], B, True)
            # inverse DFT + 1x1 mix + bias (+ GELU) in one GEMM per sample pair:
            # rows (b, o) of the pair; K = the kept modes, then the pair's 2C
            # channels against blockdiag(W, W)
            last = l == c.layers - 1
            gemm(2 * C, HW, [(kmajor(ws["Yt"], 2 * C, NR, batch_stride=2 * C * NR),
                              kmajor(self.Gm, HW, NR)),
                             (kmajor(self.pw[l], 2 * C, 2 * C),
                              mnmajor(X[l], HW, 2 * C, ld=HW, batch_stride=2 * C * HW))],
                 X[l + 1], OutMap.rowmajor(HW, batch=2 * C * HW), batch=Bp // 2,
                 row_bias=self.pw_bias[l], act=0 if last else ACT_GELU,
                 pre=None if last else ws["pre"][l], status=st)
        _lib.check("dn_fno_readout", L.dn_fno_readout(
            _c(X[c.layers]), _c(ps.P("r")), B, c.H, c.W, C, _c(ws["R"]), s))
        gemm(B * c.W, c.hidden, [(kmajor(ws["R"], B * c.W, C), kmajor(ps.B("Q1"), c.hidden, C))],
             ws["U"], OutMap.rowmajor(c.hidden), bias=ps.P("q1"), act=ACT_GELU, pre=ws["preU"],
             status=st)
        gemm(B * c.W, OUT_LD, [(kmajor(ws["U"], B * c.W, c.hidden),
                                kmajor(ps.B("Q2"), OUT_LD, c.hidden))],
             ws["out"], OutMap.rowmajor(OUT_LD), bias=ps.P("q2"), status=st)

    def _colsum(self, src, dtype, rows, cols, dst, ws):
        _lib.check("dn_colsum", self.L.dn_colsum(
            _c(src), dtype, rows, cols, cols, _c(dst), 0, _c(ws["scratch"]),
            ws["scratch"].numel(), self._stream()))

    def _channel_sums(self, d, B, dst, ws):
        """dst[c] = sum over samples and pixels of channel-first d (B, C, HW)."""
        c = self.cfg
        _lib.check("dn_fno_channel_sums", self.L.dn_fno_channel_sums(
            _c(d), B, c.width, c.H * c.W, _c(dst), _c(ws["scratch"]), self._stream()))

    def backward(self, gout_bf16: Optional[torch.Tensor] = None, B: Optional[int] = None,
                 want_input_grad: bool = False) -> Optional[torch.Tensor]:
        """Gradients of the last forward's loss into ``ps.g``.

        The loss gradient with respect to the (B*W, 8) prediction is read from
        the workspace's ``gout`` (filled by :meth:`loss`) unless given.
        Returns d loss / d eps (B, H, W) when ``want_input_grad``."""
        c, ps, L, s = self.cfg, self.ps, self.L, self._stream()
        B = B if B is not None else next(iter(self._ws))
        ws = self._bwd_workspace(B)
        if gout_bf16 is not None:
            ws["gout"].copy_(gout_bf16.view(B * c.W, OUT_LD))
        HW, C, NM, NR = c.H * c.W, c.width, c.n_modes, c.n_mode_rows
        Bp = B + (B & 1)
        st, X, part = self.status, ws["X"], ws["part"]
        F32, BF16 = 0, 2
        BW = B * c.W
        # readout MLP
        gemm(BW, c.hidden, [(kmajor(ws["gout"], BW, OUT_LD),
                             mnmajor(ps.B("Q2"), c.hidden, OUT_LD, ld=c.hidden))],
             ws["dpreU"], OutMap.rowmajor(c.hidden), act=ACT_GELU_GRAD, aux=ws["preU"], status=st)
        gemm(OUT_LD, c.hidden, [(mnmajor(ws["gout"], OUT_LD, c.W, ld=OUT_LD,
                                         batch_stride=c.W * OUT_LD),
                                 mnmajor(ws["U"], c.hidden, c.W, ld=c.hidden,
                                         batch_stride=c.W * c.hidden))],
             part, OutMap.rowmajor(c.hidden, batch=OUT_LD * c.hidden), batch=B, status=st)
        self._colsum(part, F32, B, OUT_LD * c.hidden, ps.G("Q2"), ws)
        self._colsum(ws["gout"], BF16, BW, OUT_LD, ps.G("q2"), ws)
        gemm(BW, C, [(kmajor(ws["dpreU"], BW, c.hidden), mnmajor(ps.B("Q1"), C, c.hidden, ld=C))],
             ws["dR"], OutMap.rowmajor(C), status=st)
        gemm(c.hidden, C, [(mnmajor(ws["dpreU"], c.hidden, c.W, ld=c.hidden,
                                    batch_stride=c.W * c.hidden),
                            mnmajor(ws["R"], C, c.W, ld=C, batch_stride=c.W * C))],
             part, OutMap.rowmajor(C, batch=c.hidden * C), batch=B, status=st)
        self._colsum(part, F32, B, c.hidden * C, ps.G("Q1"), ws)
        self._colsum(ws["dpreU"], BF16, BW, c.hidden, ps.G("q1"), ws)
        # readout row weights; dX_L = dpre of the last layer (no activation)
        dcur, dnext = ws["dA"], ws["dB"]
        _lib.check("dn_fno_readout_bwd", L.dn_fno_readout_bwd(
            _c(X[c.layers]), _c(ps.P("r")), _c(ws["dR"]), B, c.H, c.W, C, _c(dcur), _c(part), s))
        self._colsum(part, F32, B, c.H * C, ps.G("r"), ws)
        for l in reversed(range(c.layers)):
            # dcur = d loss / d pre_l, channel-first
            # through the inverse DFT: dY = dpre G = the analysis of dpre with
            # c/HW per kw (FwS), straight into dYm[m, ri, b, c]
            dYm = ws["dYm"]
            self._analysis(dcur, self.FwS, dYm, ws, B)
            # mode weights: rows (ri, o) of a mode are C-long runs B*C apart
            fold = dict(fold=C, fold_stride=B * C, batch_stride=2 * B * C)
            gemm(2 * C, 2 * C, [(mnmajor(dYm, 2 * C, B, ld=C, **fold),
                                 mnmajor(ws["Zm"][l], 2 * C, B, ld=C, **fold))],
                 ws["dblk"], OutMap.rowmajor(2 * C, batch=4 * C * C), batch=NM, status=st)
            _lib.check("dn_fno_unpack_mode_grads", L.dn_fno_unpack_mode_grads(
                _c(ws["dblk"]), NM, C, C, _c(ps.G(f"wre{l}")), _c(ps.G(f"wim{l}")), s))
            # back through the mixing; HW/c per mode turns G into F2^T below
            blk = self.blk[l]
            gemm(B, 2 * C, [(kmajor(dYm, B, C, batch_stride=2 * B * C),
                             mnmajor(blk, 2 * C, C, ld=2 * C, batch_stride=4 * C * C)),
                            (kmajor(dYm.view(-1)[B * C:], B, C, batch_stride=2 * B * C),
                             mnmajor(blk.view(-1)[2 * C * C:], 2 * C, C, ld=2 * C,
                                     batch_stride=4 * C * C))],
                 ws["dZm"], OutMap.rowmajor(2 * C, batch=B * 2 * C), batch=NM,
                 batch_scale=self.bscale, status=st)
            self._modes_rows(ws["dZm"], ws["dZt"], B, True)
            # 1x1 weights and bias
            gemm(C, C, [(kmajor(dcur, C, HW, batch_stride=C * HW),
                         kmajor(X[l], C, HW, batch_stride=C * HW))],
                 part, OutMap.rowmajor(C, batch=C * C), batch=B, status=st)
            self._colsum(part, F32, B, C * C, ps.G(f"W{l}"), ws)
            self._channel_sums(dcur, B, ps.G(f"b{l}"), ws)
            # dX_l = dZ F2 + W^T dpre_l (dZ F2 = (dZ diag(HW/c)) G^T), through
            # GELU of layer l-1; one GEMM per sample pair as in the forward pass
            act = ACT_GELU_GRAD if l > 0 else 0
            gemm(2 * C, HW, [(kmajor(ws["dZt"], 2 * C, NR, batch_stride=2 * C * NR),
                              kmajor(self.Gm, HW, NR)),
                             (kmajor(self.pwT[l], 2 * C, 2 * C),
                              mnmajor(dcur, HW, 2 * C, ld=HW, batch_stride=2 * C * HW))],
                 dnext, OutMap.rowmajor(HW, batch=2 * C * HW), batch=Bp // 2, act=act,
                 aux=ws["pre"][l - 1] if l > 0 else None, status=st)
            dcur, dnext = dnext, dcur
        # lift (dcur = dX0)
        gemm(C, FEAT, [(kmajor(dcur, C, HW, batch_stride=C * HW),
                        mnmajor(ws["feat"], FEAT, HW, ld=FEAT, batch_stride=HW * FEAT))],
             part, OutMap.rowmajor(FEAT, batch=C * FEAT), batch=B, status=st)
        self._colsum(part, F32, B, C * FEAT, ps.G("P"), ws)
        self._channel_sums(dcur, B, ps.G("p"), ws)
        if not want_input_grad:
            return None
        dfeat = torch.empty(B * HW, FEAT, dtype=torch.float32, device=self.dev)
        gemm(B * HW, FEAT, [(mnmajor(dcur, B * HW, C, ld=HW, fold=HW, fold_stride=C * HW),
                             mnmajor(ps.B("P"), FEAT, C, ld=FEAT))],
             dfeat, OutMap.rowmajor(FEAT), status=st)
        deps = torch.empty(B, c.H, c.W, dtype=torch.float32, device=self.dev)
        _lib.check("dn_fno_features_bwd", L.dn_fno_features_bwd(
            _c(dfeat), B * HW, c.eps_lo, c.eps_hi, _c(deps), s))
        return deps

    def loss(self, target: torch.Tensor, B: Optional[int] = None) -> torch.Tensor:
        """Mean squared error of the last forward against ``target`` (B, W,
        n_out); fills the loss gradient for :meth:`backward`.  Returns the
        loss as a device scalar (float64)."""
        c = self.cfg
        B = B if B is not None else target.shape[0]
        ws = self._bwd_workspace(B)
        tgt = torch.zeros(B * c.W, OUT_LD, dtype=torch.float32, device=self.dev)
        tgt.view(B, c.W, OUT_LD)[:, :, :c.n_out] = target.to(self.dev, torch.float32)
        n = B * c.W * c.n_out
        npart = ws["loss_part"].numel()
        _lib.check("dn_mse", self.L.dn_mse(
            _c(ws["out"]), _c(tgt), B * c.W, OUT_LD, c.n_out, 1.0 / n, _c(ws["gout"]),
            _c(ws["loss_part"]), npart, self._stream()))
        return ws["loss_part"].sum() / n

    def adam_step(self, lr: float = 1e-3, betas=(0.9, 0.999), eps: float = 1e-8,
                  weight_decay: float = 0.0) -> None:
        ps = self.ps
        ps.step += 1
        _lib.check("dn_adam", self.L.dn_adam(
            _c(ps.p), _c(ps.g), _c(ps.m), _c(ps.v), ps.n, lr, betas[0], betas[1], eps, ps.step,
            weight_decay, _c(ps.bf), self._stream()))
        self._pack()

    def check_status(self) -> None:
        v = int(self.status.item())
        if v:
            self.status.zero_()
            raise _lib.DNError("FNO GEMM", v, _lib.lib().dn_strerror(v).decode())

    def gemm_flops(self, B: int, backward: bool = True) -> float:
        """Tensor-core FLOPs the GEMMs of one forward (+ backward) execute."""
        c = self.cfg
        HW, C, NR, NM = c.H * c.W, c.width, c.n_mode_rows, c.n_modes
        M = c.modes
        # the analysis transform's two passes (W, then H)
        dft = 2 * B * C * c.H * (2 * M) * c.W + 2 * M * B * C * (4 * M) * (2 * c.H)
        fwd = 0  # the lift is a memory-bound kernel, not a GEMM
        layer = dft + 2 * NM * B * (2 * C) ** 2 + 2 * B * HW * C * (NR + C)
        fwd += c.layers * layer + 2 * B * c.W * (C * c.hidden + c.hidden * OUT_LD)
        if not backward:
            return float(fwd)
        bwd = 2 * B * c.W * (OUT_LD * c.hidden * 2 + c.hidden * C * 2)
        bwd += c.layers * (dft + 2 * 2 * NM * B * (2 * C) ** 2
                           + 2 * B * HW * C * C + 2 * B * HW * C * (NR + C))
        bwd += 2 * B * HW * C * FEAT
        return float(fwd + bwd)
