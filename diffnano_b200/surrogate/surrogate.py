"""Surrogate front end with the reference's ``NeuralSurrogate`` interface.

DiffNano's ``NeuralSurrogate`` (``diffnano/solvers/surrogate.py:78-285``)
wraps a full solver: ``train_surrogate`` generates (geometry, field) pairs
with the solver and fits a small CNN with Adam on the MSE loss
(``:135-208``), ``forward`` answers from the network except on every
``correction_interval``-th call, which runs the full solver (``:210-251``),
and ``accuracy`` compares both on fresh geometries (``:253-285``).

``FNOSurrogate`` keeps that interface with the pieces of this package: the
full solver is the batched FDTD (``FDTDLabeler``: one persistent launch per
chunk of designs), the network is the BF16 tensor-core Fourier neural
operator (``FNO2d``), training is the project's own forward/backward GEMMs
and ``dn_adam``.  Inputs are design-region permittivity maps ``(128, 128)``
(or batches of them); outputs are the complex monitor DFTs ``(L, 128)``.
"""
from __future__ import annotations

import math
import time
from typing import Dict, List, Optional

import torch

from ..solvers._result import SimResult
from .data import (FDTDLabeler, TMzSetup, from_targets, label_scale, make_dataset,
                   rel_l2_per_sample, to_targets)
from .fno import FNO2d, FNOConfig


class FNOSurrogate:
    """Fourier-neural-operator surrogate of the batched FDTD monitor DFTs.

    Parameters
    ----------
    base_solver : FDTDLabeler, optional
        The full solver (default: the 256x256 TMz set-up on ``device``).
    cfg : FNOConfig
    correction_interval : int
        Every N-th ``forward`` call runs the full solver instead (0: never).
    lr : float
        Adam learning rate.
    batch_size : int
    device : CUDA device
    seed : int
        Parameter initialisation and shuffling seed.
    """

    def __init__(self, base_solver: Optional[FDTDLabeler] = None, cfg: FNOConfig = FNOConfig(),
                 correction_interval: int = 10, lr: float = 1e-3, batch_size: int = 256,
                 device="cuda", seed: int = 0):
        self._device = torch.device(device)
        self.base_solver = base_solver or FDTDLabeler(TMzSetup(), device=self._device)
        self.cfg = cfg
        self.correction_interval = correction_interval
        self.lr = lr
        self.batch_size = batch_size
        self.seed = seed
        self.net = FNO2d(cfg, self._device, seed=seed)
        self.scale = 1.0
        self._trained = False
        self._forward_count = 0
        self.stats = {"total_predictions": 0, "total_corrections": 0}
        self.timings: Dict[str, float] = {}

    @property
    def device(self) -> torch.device:
        return self._device

    @property
    def n_wavelengths(self) -> int:
        return self.cfg.n_out // 2

    # ---- training -----------------------------------------------------------
    def train_surrogate(self, n_samples: int = 20000, n_epochs: int = 50, verbose: bool = False,
                        data_seed: int = 1, designs: Optional[torch.Tensor] = None,
                        labels: Optional[torch.Tensor] = None, schedule: str = "cosine",
                        weight_decay: float = 0.0, mirror: bool = True) -> List[float]:
        """Generate ``n_samples`` labelled designs with the full solver (unless
        ``designs``/``labels`` are given) and train; returns the per-epoch
        mean training loss.

        ``schedule``: "constant" or "cosine" (decay of the learning rate to 0
        over the run).  ``mirror``: each step flips a random half of the
        batch left-right, design and monitor line together (the set-up is
        mirror symmetric about the grid's centre column)."""
        if schedule not in ("constant", "cosine"):
            raise ValueError(f"schedule must be 'constant' or 'cosine', got {schedule!r}")
        dev = self._device
        if designs is None:
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            designs, labels = make_dataset(n_samples, data_seed, self.base_solver)
            torch.cuda.synchronize(dev)
            self.timings["label_s"] = time.perf_counter() - t0
        designs = designs.to(dev, torch.float32)
        self.scale = label_scale(labels)
        self.set_mean_label(labels.to(dev))
        targets = to_targets(labels.to(dev), self.scale)
        n = designs.shape[0]
        B = min(self.batch_size, n)
        steps = n // B
        g = torch.Generator(device=dev).manual_seed(self.seed + 17)
        history: List[float] = []
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        total = max(1, n_epochs * steps)
        it = 0
        for epoch in range(n_epochs):
            perm = torch.randperm(n, device=dev, generator=g)
            acc = torch.zeros((), dtype=torch.float64, device=dev)
            for s in range(steps):
                idx = perm[s * B:(s + 1) * B]
                x, y = designs[idx], targets[idx]
                if mirror:
                    flip = torch.rand(B, device=dev, generator=g) < 0.5
                    x = torch.where(flip[:, None, None], x.flip(-1), x)
                    y = torch.where(flip[:, None, None], y.flip(1), y)
                self.net.forward(x)
                acc += self.net.loss(y)
                self.net.ps.g.zero_()
                self.net.backward(B=B)
                lr = self.lr
                if schedule == "cosine":
                    lr = 0.5 * self.lr * (1.0 + math.cos(math.pi * it / total))
                self.net.adam_step(lr=lr, weight_decay=weight_decay)
                it += 1
            history.append(float(acc) / max(1, steps))
            if verbose and epoch % 10 == 0:
                print(f"epoch {epoch}: loss={history[-1]:.6f}")
        torch.cuda.synchronize(dev)
        self.timings["train_s"] = time.perf_counter() - t0
        self.timings["train_steps"] = n_epochs * steps
        self.net.check_status()
        self._trained = True
        return history

    # ---- inference ------------------------------------------------------------
    @torch.no_grad()
    def predict(self, eps_design: torch.Tensor) -> torch.Tensor:
        """(n, 128, 128) design eps -> complex128 (n, L, 128), batched."""
        eps = eps_design.to(self._device, torch.float32)
        if eps.dim() == 2:
            eps = eps.unsqueeze(0)
        outs = []
        for a in range(0, eps.shape[0], self.batch_size):
            part = eps[a:a + self.batch_size]
            pred = self.net.forward(part).clone()
            outs.append(from_targets(pred, self.scale, self.n_wavelengths))
        self.net.check_status()
        return torch.cat(outs)

    def forward(self, geometry: torch.Tensor, wavelengths=None, *, source=None) -> SimResult:
        """Monitor DFTs of one design (or a batch), from the network except on
        correction calls, which run the full solver."""
        if source is not None:
            raise ValueError("the surrogate is trained for one source; source must be None")
        wl = torch.tensor(self.base_solver.setup.wavelengths_nm, dtype=torch.float64)
        if wavelengths is not None:
            req = torch.as_tensor(wavelengths, dtype=torch.float64).reshape(-1)
            if req.shape != wl.shape or not torch.allclose(req, wl):
                raise ValueError(f"the surrogate predicts at {wl.tolist()} nm only")
        self._forward_count += 1
        self.stats["total_predictions"] += 1
        geo = geometry if geometry.dim() == 3 else geometry.unsqueeze(0)
        correct = not self._trained or (self.correction_interval > 0 and
                                        self._forward_count % self.correction_interval == 0)
        if correct:
            self.stats["total_corrections"] += 1
            field = self.base_solver.label(geo.to(self._device))
        else:
            field = self.predict(geo)
        return SimResult(field=field, wavelengths=wl,
                         metadata={"surrogate": not correct,
                                   "forward_count": self._forward_count})

    def accuracy(self, n_test: int = 1024, seed: int = 10_000,
                 designs: Optional[torch.Tensor] = None,
                 labels: Optional[torch.Tensor] = None) -> Dict[str, float]:
        """Held-out relative L2 error against the full solver on ``n_test``
        fresh designs, beside the error of the trivial predictor (the mean
        training-label field), which is what the method without the network
        would answer."""
        if designs is None:
            designs, labels = make_dataset(n_test, seed, self.base_solver)
        pred = self.predict(designs)
        err = rel_l2_per_sample(pred, labels.to(pred.device))
        out = {"mean_rel_l2": float(err.mean()), "median_rel_l2": float(err.median()),
               "worst_rel_l2": float(err.max()), "n_test": int(designs.shape[0])}
        if hasattr(self, "_mean_label"):
            base = rel_l2_per_sample(self._mean_label.expand_as(labels).to(pred.device),
                                     labels.to(pred.device))
            out["mean_predictor_rel_l2"] = float(base.mean())
        return out

    def set_mean_label(self, labels: torch.Tensor) -> None:
        """Record the mean training label (the no-network baseline)."""
        self._mean_label = labels.mean(dim=0, keepdim=True)

