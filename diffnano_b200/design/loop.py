"""Inverse-design loops: plain FDTD Adam, and surrogate-assisted (the
surrogate proposes and prescreens, the FDTD verifies and judges).

The reference's two-stage driver (``diffnano/solvers/proxy_prescreen.py:147-274``,
``TwoStageOptimizer``: generate candidates, rank them with a fast proxy,
evaluate the top ones with the full solver) is the pattern; here it runs
inside a gradient loop:

* :func:`plain_loop` -- every iteration evaluates the design with the 3-D FDTD
  forward + adjoint and takes an Adam step on the density (``dn_adam``), with
  the projection sharpness beta raised from ``beta[0]`` to ``beta[1]``
  (``beta_continuation_schedule``).
* :class:`SurrogateAssistedLoop` -- a Fourier neural operator S trained on the
  2-D proxy (labelled by the batched FDTD) is corrected to first order at the
  accepted design rho_k (model m(rho) = f_k + S(rho) - S(rho_k) + (g_k -
  grad S(rho_k)) . (rho - rho_k), which matches the FDTD value f_k and
  gradient g_k there: first-order model management, Alexandrov et al.,
  Structural Optimization 15, 1998).  Adam on m from rho_k (beta ramped to the
  next outer value) proposes a path; ``n_candidates`` snapshots of it are
  ranked by m in one batched inference and the best goes to the 3-D FDTD
  forward + adjoint.  It is accepted when its FDTD figure of merit does not
  fall more than ``tolerance`` below the last accepted one; otherwise the loop
  falls back to a plain Adam step from rho_k with g_k.  The inner step size is
  a trust region: doubled when the FDTD gain is at least 3/4 of the predicted
  one, quartered on a rejection.  Every verified sample also fine-tunes the
  network.  Wall time includes the proxy labelling and the training.
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
from .metalens import Metalens3D, Proxy2D, proxy_dataset
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
    """Output-space map from the cross-section model to the 3-D focal field.

    The 3-D lens is finite in y and the plane wave also passes beside it, so
    the 3-D focal field is not the 2-D cross-section's; measured over very
    different designs (uniform, random, cross-section optima) it is close to
    an affine image of it, E3 = c S + b with complex c and b (7.6 % relative
    residual over 13 designs, against 9.7 % for E3 = c S).  The map is fitted
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
    kind: str  # "adam", "surrogate", "fallback"
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
    n_train: int = 4096
    epochs: int = 20
    batch: int = 256
    lr: float = 1e-3
    n_candidates: int = 32
    inner_steps: int = 32
    inner_lr: float = 0.02
    max_inner_lr: float = 0.16
    min_inner_lr: float = 1e-4
    outer_schedule: int = 10  # outer iterations over which beta reaches its end value
    max_verify: int = 40
    tolerance: float = 0.02
    ft_steps: int = 10
    ft_lr: float = 2e-4
    fallback_lr: float = 0.02
    seed: int = 0
    fno: FNOConfig = field(default_factory=lambda: FNOConfig(H=40, W=256, eps_lo=1.0,
                                                             eps_hi=12.1))


class SurrogateAssistedLoop:
    def __init__(self, problem: Metalens3D, cfg: SurrogateConfig = SurrogateConfig(),
                 proxy: Optional[Proxy2D] = None):
        self.problem = problem
        self.cfg = cfg
        s = problem.setup
        if (cfg.fno.H, cfg.fno.W) != s.design_shape:
            raise ValueError(f"surrogate input {(cfg.fno.H, cfg.fno.W)} != design {s.design_shape}")
        self.proxy = proxy or Proxy2D(s, device=problem.device)
        self.net = FNO2d(cfg.fno, problem.device, seed=cfg.seed)
        self.scale = 1.0
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
        self._heldout = proxy_dataset(self.proxy, 256, seed=c.seed + 999)

    def proxy_error(self) -> float:
        """Mean relative L2 error of the network on 256 held-out proxy designs."""
        from ..surrogate.data import rel_l2_per_sample
        eps, labels = self._heldout
        pred = from_targets(self.net.forward(eps).clone(), self.scale, labels.shape[1])
        return float(rel_l2_per_sample(pred, labels).mean())

    def _focal(self, pred: torch.Tensor) -> torch.Tensor:
        s = self.problem.setup
        li, fc = s.center_index, s.focus_col
        return pred[:, fc, 2 * li] ** 2 + pred[:, fc, 2 * li + 1] ** 2

    def predict_fom(self, eps_design: torch.Tensor) -> torch.Tensor:
        return self._focal(self.net.forward(eps_design)) * self.scale ** 2

    def _value_grad(self, rho: torch.Tensor, beta: float):
        """Surrogate focal intensity S(rho) and dS/drho (FOM units)."""
        s = self.problem.setup
        W = s.design_shape[1]
        li, fc = s.center_index, s.focus_col
        x = rho.detach().clone().requires_grad_(True)
        eps = s.eps_design(x, beta).unsqueeze(0)
        pred = self.net.forward(eps.detach())
        value = self._focal(pred)[0] * self.scale ** 2
        gout = torch.zeros(W, OUT_LD, device=x.device)
        gout[fc, 2 * li] = -2.0 * pred[0, fc, 2 * li]
        gout[fc, 2 * li + 1] = -2.0 * pred[0, fc, 2 * li + 1]
        self.net._bwd_workspace(1)["gout"].copy_(gout.to(torch.bfloat16))
        deps = self.net.backward(B=1, want_input_grad=True)  # d(-S/scale^2)/d eps
        eps.backward(deps)
        return float(value), -x.grad * self.scale ** 2

    def _ascent(self, rho: torch.Tensor, b0: float, b1: float, corr: torch.Tensor,
                steps: int, lr: float, fom_ref: float) -> List[torch.Tensor]:
        """Adam (learning rate ``lr``) on the corrected model m = S + corr .
        (rho - rho_k); density snapshots along the path (the candidates)."""
        c = self.cfg
        opt = DensityAdam(rho, lr)
        every = max(1, steps // c.n_candidates)
        snaps = []
        for k in range(steps):
            b = b0 * (b1 / b0) ** ((k + 1) / steps)
            _, dS = self._value_grad(opt.rho, b)
            opt.ascend(dS + corr, 1.0 / fom_ref)
            if (k + 1) % every == 0:
                snaps.append(opt.rho.clone())
        return snaps[-c.n_candidates:]

    def _fine_tune(self) -> None:
        c = self.cfg
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

    def _record_sample(self, eps_design: torch.Tensor, dft_line: torch.Tensor) -> None:
        self._buf_x.append(eps_design.detach().to(torch.float32))
        self._buf_y.append(to_targets(dft_line.unsqueeze(0), self.scale)[0])

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
        rho = rho0.to(dev, torch.float32).clone()
        b = beta[0]
        fom, grad, dft = p.evaluate(rho, b, grad=True)
        self._record_sample(s.eps_design(rho, b).detach(), dft)
        hist.append(Record(1, time.perf_counter() - t0, fom, b, "start"))
        fallback = DensityAdam(rho, c.fallback_lr)
        fom0 = fom
        reached = None
        steps = c.inner_steps
        lr = c.inner_lr  # trust region: the inner path's step size
        o = 0
        while len(hist) < c.max_verify:
            o += 1
            b_next = beta_continuation_schedule(o, c.outer_schedule, beta[0], beta[1])
            # first-order correction: the model matches the FDTD value and
            # gradient at the accepted design
            s0, dS0 = self._value_grad(rho, b)
            corr = grad - dS0
            snaps = self._ascent(rho, b, b_next, corr, steps, lr, fom0)
            with torch.no_grad():
                eps_c = torch.stack([s.eps_design(r, b_next) for r in snaps])
                S = self.predict_fom(eps_c)
                lin = torch.stack([(corr * (r - rho)).sum() for r in snaps])
                model = fom + (S - s0) + lin
            best = int(torch.argmax(model))
            cand = snaps[best]
            f_new, g_new, dft_new = p.evaluate(cand, b_next, grad=True)
            self._record_sample(eps_c[best], dft_new)
            ok = f_new >= (1.0 - c.tolerance) * fom
            hist.append(Record(len(hist) + 1, time.perf_counter() - t0, f_new, b_next,
                               "surrogate", ok))
            predicted = float(model[best])
            cand_stats.append({"model_best": predicted, "fdtd": f_new, "fom_before": fom,
                               "inner_lr": lr, "pick": best})
            gain_pred = predicted - fom
            ratio = (f_new - fom) / gain_pred if gain_pred > 0 else 0.0
            if ok:
                rho, fom, grad, b = cand.clone(), f_new, g_new, b_next
                if ratio > 0.75:
                    lr = min(c.max_inner_lr, 2.0 * lr)
            else:
                lr = max(c.min_inner_lr, 0.25 * lr)
                # plain step from the accepted design with its FDTD gradient
                fallback.rho.copy_(rho)
                r2 = fallback.ascend(grad, 1.0 / fom0).clone()
                f2, g2, d2 = p.evaluate(r2, b_next, grad=True)
                self._record_sample(s.eps_design(r2, b_next).detach(), d2)
                hist.append(Record(len(hist) + 1, time.perf_counter() - t0, f2, b_next,
                                   "fallback"))
                rho, fom, grad, b = r2, f2, g2, b_next
            self._fine_tune()
            if target is not None and b >= beta[1] * (1 - 1e-9) and fom >= 0.99 * target:
                reached = time.perf_counter() - t0
                break
        torch.cuda.synchronize(dev)
        at_end = [r.fom for r in hist if r.beta >= beta[1] * (1 - 1e-9)]
        return {"rho": rho, "history": hist, "final_fom": fom,
                "best_fom": max(at_end) if at_end else None,
                "wall_s": time.perf_counter() - t0, "time_to_target_s": reached,
                "verifications": p.evaluations, "timings": dict(self.timings),
                "candidates": cand_stats, "fom0": fom0}
