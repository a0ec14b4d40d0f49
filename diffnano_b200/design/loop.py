"""Inverse-design loops: plain FDTD Adam, and surrogate-assisted (a learned
surrogate prescreens, the 3-D FDTD verifies and judges).

The reference's two-stage driver (``diffnano/solvers/proxy_prescreen.py:147-274``,
``TwoStageOptimizer``: generate candidates, rank them with a fast proxy,
evaluate the top ones with the full solver) and its multi-fidelity designer
(``diffnano/design/multifidelity.py:277-470``: screen cheaply, verify the top
ones expensively) are the pattern; here they run inside a gradient loop:

* :func:`plain_loop` -- every iteration evaluates the design with the 3-D FDTD
  forward + adjoint and takes an Adam step on the density (``dn_adam``), with
  the projection sharpness beta raised from ``beta[0]`` to ``beta[1]``
  (``beta_continuation_schedule``).
* :class:`SurrogateAssistedLoop` -- candidates proposed by a cheaper model of
  the lens (by default the same 3-D problem on 2x coarser cells; or the 2-D
  cross-section), mapped to the 3-D focal field by :class:`OutputMap`, ranked
  by a Fourier neural operator trained on batched-FDTD labels, checked by the
  model, verified by the 3-D FDTD.  Wall time includes the proxy labelling
  and the network's training.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import torch

from .. import _lib
from ..surrogate.data import from_targets, label_scale, to_targets
from ..surrogate.fno import FNO2d, FNOConfig, OUT_LD
from .metalens import Metalens3D, Proxy2D, coarse_model, proxy_dataset
from .projection import beta_continuation_schedule


class DensityAdam:
    """Adam ascent on a density in [0, 1] with the ``dn_adam`` kernel."""

    def __init__(self, rho: torch.Tensor, lr: float):
        self.rho = rho.detach().to(torch.float32).contiguous().clone()
        self.g = torch.zeros_like(self.rho)
        self.m = torch.zeros_like(self.rho)
        self.v = torch.zeros_like(self.rho)
        self.lr = lr
        self.t = 0

    def ascend(self, grad: torch.Tensor, scale: float = 1.0) -> torch.Tensor:
        """One step up ``grad`` (scaled by ``scale``); returns the new density."""
        self.t += 1
        torch.mul(grad.to(self.g.dtype), -scale, out=self.g)
        _lib.check("dn_adam", _lib.lib().dn_adam(
            self.rho.data_ptr(), self.g.data_ptr(), self.m.data_ptr(), self.v.data_ptr(),
            self.rho.numel(), self.lr, 0.9, 0.999, 1e-8, self.t, 0.0, None,
            ctypes.c_void_p(torch.cuda.current_stream(self.rho.device).cuda_stream)))
        self.rho.clamp_(0.0, 1.0)
        return self.rho


class OutputMap:
    """Output-space map from a cheaper model's focal value to the 3-D focal field.

    For the 2-D cross-section: the 3-D lens is finite in y and the plane wave
    also passes beside it, so the 3-D focal field is not the cross-section's;
    measured over very different designs (uniform, random, cross-section
    optima) it is close to an affine image of it, E3 = c S + b with complex c
    and b (7.6 % relative residual over 13 designs, against 9.7 % for E3 =
    c S).  The same form maps the coarse 3-D model and the network.  The map is fitted
    by complex least squares to the (surrogate value, FDTD value) pairs of
    every 3-D verification so far: with one pair b = 0 and c = E3 / S; with
    more, both (Bandler et al.'s output space mapping, IEEE MTT 52, 2004)."""

    def __init__(self):
        self.s: List[complex] = []
        self.e: List[complex] = []

    def add(self, s: complex, e: complex) -> None:
        self.s.append(complex(s))
        self.e.append(complex(e))

    def coef(self):
        if not self.s:
            return 1.0 + 0.0j, 0.0j
        if len(self.s) == 1:
            s0 = self.s[0] if abs(self.s[0]) > 0 else 1.0
            return self.e[0] / s0, 0.0j
        S = torch.tensor(self.s, dtype=torch.complex128)
        E = torch.tensor(self.e, dtype=torch.complex128)
        A = torch.stack([S, torch.ones_like(S)], 1)
        sol = torch.linalg.lstsq(A, E[:, None]).solution[:, 0]
        return complex(sol[0]), complex(sol[1])

    def residual(self) -> float:
        """Relative residual of the current fit over its pairs."""
        if len(self.s) < 2:
            return 0.0
        c, b = self.coef()
        num = sum(abs(c * s + b - e) ** 2 for s, e in zip(self.s, self.e))
        return math.sqrt(num / sum(abs(e) ** 2 for e in self.e))


@dataclass
class Record:
    verification: int
    wall_s: float
    fom: float
    beta: float
    kind: str  # "adam" (plain loop); "start", "warm start", "surrogate" (assisted loop)
    accepted: bool = True


def plain_loop(problem: Metalens3D, rho0: torch.Tensor, iters: int = 100, lr: float = 0.02,
               beta=(1.0, 32.0)) -> Dict:
    """Adam on the FDTD gradient for ``iters`` iterations."""
    dev = problem.device
    opt = DensityAdam(rho0.to(dev), lr)
    hist: List[Record] = []
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    fom0 = None
    for k in range(iters):
        b = beta_continuation_schedule(k, max(1, iters - 1), beta[0], beta[1])
        fom, g, _ = problem.evaluate(opt.rho, b, grad=True)
        fom0 = fom0 or fom
        hist.append(Record(k + 1, time.perf_counter() - t0, fom, b, "adam"))
        if k < iters - 1:
            opt.ascend(g, 1.0 / fom0)
    torch.cuda.synchronize(dev)
    return {"rho": opt.rho.clone(), "history": hist, "final_fom": hist[-1].fom,
            "best_fom": max(r.fom for r in hist), "wall_s": time.perf_counter() - t0,
            "fom0": fom0}


@dataclass
class SurrogateConfig:
    n_train: int = 1024          # proxy designs labelled by the batched 2-D FDTD
    epochs: int = 12
    batch: int = 256
    lr: float = 1e-3
    model: str = "coarse3d"      # proposing model: "coarse3d" or "cross-section"
    coarse_factor: int = 2       # cell-size factor of the coarse 3-D model
    warm_steps: int = 100        # warm start: Adam steps on the mapped model, beta ramped
    warm_lr: float = 0.02
    tr_beta_frac: float = 0.5    # < 1: the warm start stops at this fraction of the end
    tr_beta_steps: int = 8       # beta; the first tr_beta_steps verifications raise it
    inner_steps: int = 8         # trust-region path per verification (one snapshot per step)
    n_scales: int = 4            # step-length variants per snapshot: candidates = steps * scales
    n_check: int = 2             # candidates the FNO passes on to the model's check
    inner_lr: float = 0.02
    max_inner_lr: float = 0.2
    min_inner_lr: float = 1e-4
    max_verify: int = 60
    ft_steps: int = 5
    ft_lr: float = 2e-4
    seed: int = 0
    fno: FNOConfig = field(default_factory=lambda: FNOConfig(H=40, W=256, eps_lo=1.0,
                                                             eps_hi=12.1))

    @property
    def n_candidates(self) -> int:
        return self.inner_steps * self.n_scales


class SurrogateAssistedLoop:
    """Surrogate-assisted design loop: the 3-D FDTD judges every accepted step.

    Three models of the FOM, cheapest first:

    * the FNO (trained on batched-FDTD labels of the lens's 2-D cross-section)
      prescreens ``n_candidates`` candidate steps per verification in one
      batched inference and passes ``n_check`` on; its focal value is mapped
      to the 3-D focal field by its own :class:`OutputMap`, fitted to every
      verification so far;
    * the proposing model, mapped to the 3-D focal field by an
      :class:`OutputMap`: by default (``model="coarse3d"``) the same lens on
      2x coarser cells (:func:`coarse_model`, ~0.28 s for a value and its
      adjoint gradient on the workload, ~1/11 of the full solve), or the 2-D
      cross-section (``"cross-section"``, ~0.07 s; its optimum is about half
      the 3-D one); it proposes the steps and checks the prescreened
      candidates;
    * the 3-D FDTD forward + adjoint verifies the best checked candidate.

    Run: (1) the 3-D FOM at the start design (forward only); (2) warm start:
    Adam on the mapped model with beta ramped to ``tr_beta_frac`` of its end
    value, verified in 3-D; (3) trust-region steps, the first
    ``tr_beta_steps`` of them raising beta geometrically to its end value
    (every step taken while beta rises, as the plain loop takes every step;
    at beta 32 the landscape admits only tiny steps, so the design is shaped
    while it is still grey): the model corrected to first
    order at the accepted design rho_k, m(rho) = f_k + M(rho) - M(rho_k) +
    (g_k - grad M(rho_k)) . (rho - rho_k), which matches the 3-D value and
    gradient there (first-order model management, Alexandrov et al.,
    Structural Optimization 15, 1998); Adam on m gives ``inner_steps``
    snapshots, each at ``n_scales`` step lengths; the FNO ranks them, the
    model checks the top ``n_check``, the best goes to 3-D.  Accepted when its
    FOM does not fall; the step size doubles when the gain reaches 3/4 of the
    predicted one, halves when it falls below 1/4 of it or the step is
    rejected (the usual trust-region ratio test).  Wall time includes the proxy
    labelling and the network's training.

    Measured on the 384x384x192 workload: the cross-section model saturates
    near x47 of the start's 3-D FOM, the coarse 3-D model's own optimum scores
    x68-69 on the full grid; the network (held-out error ~0.7 on the
    cross-section labels) cannot propose designs itself (ascending its own
    prediction leads to designs it overrates by orders of magnitude), so it
    only ranks.
    """

    def __init__(self, problem: Metalens3D, cfg: SurrogateConfig = SurrogateConfig(),
                 proxy: Optional[Proxy2D] = None):
        self.problem = problem
        self.cfg = cfg
        s = problem.setup
        if (cfg.fno.H, cfg.fno.W) != s.design_shape:
            raise ValueError(f"surrogate input {(cfg.fno.H, cfg.fno.W)} != design {s.design_shape}")
        if cfg.model not in ("coarse3d", "cross-section"):
            raise ValueError(f"model must be 'coarse3d' or 'cross-section', got {cfg.model!r}")
        self.proxy = proxy or Proxy2D(s, device=problem.device)
        self.model = (coarse_model(s, cfg.coarse_factor, problem.device)
                      if cfg.model == "coarse3d" else self.proxy)
        self.net = FNO2d(cfg.fno, problem.device, seed=cfg.seed)
        self.scale = 1.0
        self.map = OutputMap()    # model focal value -> 3-D focal field
        self.nmap = OutputMap()   # network focal value -> 3-D focal field
        self.timings: Dict[str, float] = {}
        self._buf_x: List[torch.Tensor] = []
        self._buf_y: List[torch.Tensor] = []

    # ---- surrogate ------------------------------------------------------------
    def prepare(self) -> None:
        """Label the proxy training set with the batched 2-D FDTD and train."""
        c, dev = self.cfg, self.problem.device
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        eps, labels = proxy_dataset(self.proxy, c.n_train, seed=c.seed + 100)
        torch.cuda.synchronize(dev)
        t1 = time.perf_counter()
        self.scale = label_scale(labels)
        tgt = to_targets(labels, self.scale)
        n, B = eps.shape[0], min(c.batch, eps.shape[0])
        g = torch.Generator(device=dev).manual_seed(c.seed + 7)
        total, it = max(1, c.epochs * (n // B)), 0
        for _ in range(c.epochs):
            perm = torch.randperm(n, device=dev, generator=g)
            for s in range(n // B):
                idx = perm[s * B:(s + 1) * B]
                self.net.forward(eps[idx])
                self.net.loss(tgt[idx])
                self.net.ps.g.zero_()
                self.net.backward(B=B)
                self.net.adam_step(lr=0.5 * c.lr * (1 + math.cos(math.pi * it / total)))
                it += 1
        torch.cuda.synchronize(dev)
        self.net.check_status()
        self.timings.update(label_s=t1 - t0, train_s=time.perf_counter() - t1)

    def proxy_error(self) -> float:
        """Mean relative L2 error of the network on 256 held-out proxy designs
        (labelled on first use, outside the timed loop)."""
        from ..surrogate.data import rel_l2_per_sample
        if getattr(self, "_heldout", None) is None:
            self._heldout = proxy_dataset(self.proxy, 256, seed=self.cfg.seed + 999)
        eps, labels = self._heldout
        pred = from_targets(self.net.forward(eps).clone(), self.scale, labels.shape[1])
        return float(rel_l2_per_sample(pred, labels).mean())

    def _fno_focal(self, eps_design: torch.Tensor) -> torch.Tensor:
        """Network's complex focal value (centre wavelength) for a batch."""
        s = self.problem.setup
        li, fc = s.center_index, s.focus_col
        pred = self.net.forward(eps_design)
        return torch.complex(pred[:, fc, 2 * li].double(),
                             pred[:, fc, 2 * li + 1].double()) * self.scale

    def _fine_tune(self) -> None:
        c = self.cfg
        if not self._buf_x:
            return
        X = torch.stack(self._buf_x)
        Y = torch.stack(self._buf_y)
        n = X.shape[0]
        B = min(16, n)
        g = torch.Generator(device=X.device).manual_seed(len(self._buf_x))
        for _ in range(c.ft_steps):
            idx = torch.randperm(n, device=X.device, generator=g)[:B]
            self.net.forward(X[idx])
            self.net.loss(Y[idx])
            self.net.ps.g.zero_()
            self.net.backward(B=B)
            self.net.adam_step(lr=c.ft_lr)

    # ---- models -------------------------------------------------------------------
    def _mapped(self, rho: torch.Tensor, beta: float, grad: bool):
        """(model focal value, mapped intensity M, dM/drho)."""
        cc, bb = self.map.coef()
        return self.model.focal(rho, beta, cc, bb, grad=grad)

    def _check(self, cands: torch.Tensor, eps_c: torch.Tensor, beta: float) -> torch.Tensor:
        """Model focal values of the prescreened candidates (complex128)."""
        s = self.problem.setup
        if self.cfg.model == "cross-section":
            labels = self.proxy.label(eps_c)  # one batched cross-section FDTD launch
            for e_, l_ in zip(eps_c, labels):
                self._buf_x.append(e_.float())
                self._buf_y.append(to_targets(l_.unsqueeze(0), self.scale)[0])
            return labels[:, s.center_index, s.focus_col]
        vals = [self.model.focal(r, beta)[0] for r in cands]
        return torch.tensor(vals, dtype=torch.complex128, device=cands.device)

    def _verify(self, rho: torch.Tensor, beta: float, grad: bool = True):
        """3-D FDTD forward (+ adjoint): (FOM, gradient, complex focal value)."""
        s = self.problem.setup
        f, g, dft = self.problem.evaluate(rho, beta, grad=grad)
        return f, g, complex(dft[s.center_index, s.focus_col])

    def _pair(self, rho: torch.Tensor, beta: float, e3: complex, e_model: complex) -> None:
        """Add a verified design's focal values to both output maps."""
        self.map.add(e_model, e3)
        with torch.no_grad():
            e_net = complex(self._fno_focal(self.problem.setup.eps_design(rho, beta)[None])[0])
        self.nmap.add(e_net, e3)

    # ---- loop -------------------------------------------------------------------
    def run(self, rho0: torch.Tensor, target: Optional[float] = None,
            beta=(1.0, 32.0)) -> Dict:
        c, p, s = self.cfg, self.problem, self.problem.setup
        dev = p.device
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        self.prepare()
        hist: List[Record] = []
        cand_stats = []
        reached = None
        b_end = beta[1]

        def done(fom, b):
            return target is not None and b >= b_end * (1 - 1e-9) and fom >= 0.99 * target

        # (1) the start design (its FOM is the reference of the step scale)
        rho = rho0.to(dev, torch.float32).clone()
        fom, _, e3 = self._verify(rho, beta[0], grad=False)
        fom0 = fom
        e_m, _, _ = self.model.focal(rho, beta[0])
        self._pair(rho, beta[0], e3, e_m)
        hist.append(Record(1, time.perf_counter() - t0, fom, beta[0], "start"))
        # (2) warm start on the mapped model, beta ramped to b_w (a fraction of
        # the end value; the trust-region steps finish the ramp)
        b_w = max(beta[0], b_end * c.tr_beta_frac) if 0.0 < c.tr_beta_frac < 1.0 else b_end
        opt = DensityAdam(rho, c.warm_lr)
        _, m_ref, _ = self._mapped(rho, beta[0], grad=False)
        for k in range(c.warm_steps):
            b = beta[0] * (b_w / beta[0]) ** (k / max(1, c.warm_steps - 1))
            _, _, gm = self._mapped(opt.rho, b, grad=True)
            opt.ascend(gm, 1.0 / max(m_ref, 1e-30))
        cand = opt.rho.clone()
        f_w, g_w, e3_w = self._verify(cand, b_w)
        e_mw, _, _ = self.model.focal(cand, b_w)
        self._pair(cand, b_w, e3_w, e_mw)
        hist.append(Record(2, time.perf_counter() - t0, f_w, b_w, "warm start"))
        # the start was judged at beta[0]; the warm start is the new base
        b = b_w
        n_tr = 0
        rho, fom, grad = cand, f_w, g_w
        if done(fom, b):
            reached = time.perf_counter() - t0
        lr = c.inner_lr
        # (3) trust-region steps on the corrected model
        while reached is None and len(hist) < c.max_verify:
            # beta of this verification: raised geometrically to the end value
            # over tr_beta_steps verifications when the warm start stopped short
            b_prev = b
            n_tr += 1
            if b < b_end:
                b = min(b_end, b_w * (b_end / b_w) ** (n_tr / max(1, c.tr_beta_steps)))
            ramping = b > b_prev
            e_k, m_k, dm_k = self._mapped(rho, b, grad=True)
            corr = grad - dm_k
            inner = DensityAdam(rho, lr)
            snaps = []
            for _ in range(c.inner_steps):
                _, _, dm = self._mapped(inner.rho, b, grad=True)
                inner.ascend(dm + corr, 1.0 / fom0)
                snaps.append(inner.rho.clone())
            scales = torch.linspace(0.5, 2.0, c.n_scales).tolist()
            cands = torch.stack([(rho + sc * (sn - rho)).clamp(0.0, 1.0)
                                 for sn in snaps for sc in scales])
            lin = ((cands - rho) * corr).flatten(1).sum(1).double()
            cc, bb = self.map.coef()
            cn, bn = self.nmap.coef()
            with torch.no_grad():
                eps_c = torch.stack([s.eps_design(r, b) for r in cands])
                fno_e = self._fno_focal(eps_c)
                fno_k = self._fno_focal(s.eps_design(rho, b).unsqueeze(0))[0]
                pre = fom + ((cn * fno_e + bn).abs() ** 2 - abs(cn * fno_k + bn) ** 2) + lin
                top = torch.topk(pre, min(c.n_check, len(cands))).indices
                e_top = self._check(cands[top], eps_c[top], b)
            model = fom + ((cc * e_top + bb).abs() ** 2 - m_k) + lin[top]
            j = int(torch.argmax(model))
            pick = int(top[j])
            f_new, g_new, e3_new = self._verify(cands[pick], b)
            self._pair(cands[pick], b, e3_new, complex(e_top[j]))
            # while beta rises the FOMs of consecutive steps are not comparable:
            # every step is taken (as the plain loop takes every step)
            ok = ramping or f_new >= fom
            hist.append(Record(len(hist) + 1, time.perf_counter() - t0, f_new, b, "surrogate",
                               ok))
            predicted = float(model[j])
            cand_stats.append({"predicted": predicted, "fdtd": f_new, "fom_before": fom,
                               "lr": lr, "pick": pick, "fno_rank_of_pick": int(j),
                               "map_residual": self.map.residual()})
            # trust-region ratio: achieved / predicted gain
            ratio = (f_new - fom) / (predicted - fom) if predicted > fom else 0.0
            if ok and ratio >= 0.75:
                lr = min(c.max_inner_lr, 2.0 * lr)
            elif not ok or ratio < 0.25:
                lr = max(c.min_inner_lr, 0.5 * lr)
            if ok:
                rho, fom, grad = cands[pick].clone(), f_new, g_new
            if c.model == "cross-section":
                self._fine_tune()
            if done(fom, b):
                reached = time.perf_counter() - t0
        torch.cuda.synchronize(dev)
        at_end = [r.fom for r in hist if r.beta >= b_end * (1 - 1e-9)]
        return {"rho": rho, "history": hist, "final_fom": fom,
                "best_fom": max(at_end) if at_end else None,
                "wall_s": time.perf_counter() - t0, "time_to_target_s": reached,
                "verifications": p.evaluations, "timings": dict(self.timings),
                "candidates": cand_stats, "fom0": fom0, "model": c.model,
                "map": {"coef": [str(v) for v in self.map.coef()],
                        "residual": self.map.residual()},
                "net_map": {"coef": [str(v) for v in self.nmap.coef()],
                            "residual": self.nmap.residual()}}
