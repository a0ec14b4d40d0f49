"""Training data for the surrogate, generated by the batched FDTD.

Designs are seeded binary Si/SiO2 blob maps (N(0,1) noise, Gaussian filter of
sigma drawn from [2, 6] cells, threshold 0 -- the blob recipe of the 256x256
TMz workload) placed in the central 128x128 region of a 256x256 SiO2 grid.
Each design is labelled with the complex DFT of Ez on the central 128 cells of
the monitor row at three wavelengths, computed by ``FDTDBatch2D`` (one
persistent launch per chunk of designs) with the workload's set-up: dx = 20
nm, 20-cell CPML, Courant 0.5, 2000 steps, Gaussian-pulse line source at row
30 (1.55 um centre, 0.2 um width), monitor row 226 at 1.50 / 1.55 / 1.60 um.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Sequence, Tuple

import torch
import torch.nn.functional as F

from ..solvers.batch2d import BatchInstance, FDTDBatch2D
from ..workloads import EPS_SI, EPS_SIO2, gaussian_pulse_for_band

SIGMA_STEP = 0.25  # filter widths are drawn on this grid so designs batch by kernel


@dataclass(frozen=True)
class TMzSetup:
    side: int = 256
    design: int = 128
    dl: float = 20.0
    pml: int = 20
    courant: float = 0.5
    n_steps: int = 2000
    src_row: int = 30
    mon_row: int = 226
    wavelengths_nm: Tuple[float, ...] = (1500.0, 1550.0, 1600.0)
    center_nm: float = 1550.0
    bandwidth_nm: float = 200.0

    @property
    def offset(self) -> int:
        return (self.side - self.design) // 2

    def instance(self) -> BatchInstance:
        src = gaussian_pulse_for_band(self.center_nm, self.bandwidth_nm)
        src.update(row=self.src_row)
        return BatchInstance(grid_shape=(self.side, self.side), n_steps=self.n_steps, dl=self.dl,
                             wavelength_nm=self.center_nm, pml_layers=self.pml,
                             courant=self.courant, source=src,
                             monitor={"row": self.mon_row,
                                      "wavelengths_nm": list(self.wavelengths_nm)})


def _gauss_kernel(sigma: float, dtype) -> torch.Tensor:
    # the workload filter: radius 2*sigma, 2r+1 taps (odd), sigma = r/2
    r = 2.0 * sigma
    k = int(2 * r + 1)
    if k % 2 == 0:
        k += 1
    t = torch.arange(k, dtype=dtype) - k // 2
    g = torch.exp(-(t ** 2) / (2 * sigma ** 2))
    return g / g.sum()


def blob_designs(n: int, seed: int, sigma_range=(2.0, 6.0), size: int = 128,
                 device="cpu") -> Tuple[torch.Tensor, torch.Tensor]:
    """``n`` seeded 0/1 blob maps ``(n, size, size)`` (float32) and their
    filter sigmas.  Filtering runs grouped by sigma (separable, zero padded)."""
    g = torch.Generator().manual_seed(seed)
    noise = torch.randn(n, size, size, dtype=torch.float32, generator=g)
    steps = int(round((sigma_range[1] - sigma_range[0]) / SIGMA_STEP))
    idx = torch.randint(0, steps + 1, (n,), generator=g)
    sigmas = sigma_range[0] + SIGMA_STEP * idx.to(torch.float64)
    noise = noise.to(device)
    out = torch.empty(n, size, size, dtype=torch.float32, device=device)
    for v in torch.unique(idx).tolist():
        sel = (idx == v).nonzero().flatten().to(device)
        ker = _gauss_kernel(float(sigma_range[0] + SIGMA_STEP * v), torch.float32).to(device)
        k = ker.numel()
        x = noise[sel].unsqueeze(1)
        x = F.conv2d(x, ker.view(1, 1, 1, k), padding=(0, k // 2))
        x = F.conv2d(x, ker.view(1, 1, k, 1), padding=(k // 2, 0))
        out[sel] = (x[:, 0] > 0).to(torch.float32)
    return out, sigmas


def design_eps(masks: torch.Tensor) -> torch.Tensor:
    """0/1 design maps -> design-region permittivity (Si where 1, SiO2 where 0)."""
    return EPS_SIO2 + (EPS_SI - EPS_SIO2) * masks


class FDTDLabeler:
    """Labels design-region permittivity maps with monitor DFTs by running the
    batched FDTD on chunks of ``chunk`` designs (one persistent launch each)."""

    def __init__(self, setup: TMzSetup = TMzSetup(), chunk: int = 2048, device="cuda"):
        self.setup = setup
        self.chunk = chunk
        self.device = torch.device(device)
        self._batch = None
        self._n = 0
        self.cell_steps = 0

    def _solver(self, n: int) -> FDTDBatch2D:
        if self._batch is None or self._n != n:
            # a chunk of 2048 256^2 grids streams ~3.7 GB per step: the persistent
            # strip-march kernel (32-row tiles) labels it faster than one
            # thread-block cluster per grid (129 vs 118 Gcell/s, identical DFTs)
            self._batch = FDTDBatch2D([self.setup.instance() for _ in range(n)], "TM",
                                      torch.float32, self.device, tile_rows=32, cluster=False)
            self._n = n
        return self._batch

    def full_eps(self, eps_design: torch.Tensor) -> torch.Tensor:
        s = self.setup
        n = eps_design.shape[0]
        eps = torch.full((n, s.side, s.side), EPS_SIO2, dtype=torch.float64, device=self.device)
        o = s.offset
        eps[:, o:o + s.design, o:o + s.design] = eps_design.to(self.device, torch.float64)
        return eps

    @torch.no_grad()
    def label(self, eps_design: torch.Tensor) -> torch.Tensor:
        """(n, 128, 128) design eps -> complex128 (n, n_wavelengths, 128)."""
        s = self.setup
        out = []
        for a in range(0, eps_design.shape[0], self.chunk):
            part = eps_design[a:a + self.chunk]
            n = part.shape[0]
            batch = self._solver(n)
            eps = self.full_eps(part)
            _, dfts = batch.run_forward(eps)
            batch.check_status()
            d = torch.stack([x[:, 0, s.offset:s.offset + s.design] for x in dfts])
            out.append(d)
            self.cell_steps += n * s.side * s.side * s.n_steps
        return torch.cat(out)


def to_targets(labels: torch.Tensor, scale: float) -> torch.Tensor:
    """complex (n, L, P) -> real (n, P, 2L) ordered (re, im) per wavelength, / scale."""
    r = torch.view_as_real(labels)  # (n, L, P, 2)
    return (r.permute(0, 2, 1, 3).reshape(labels.shape[0], labels.shape[2], -1) / scale).to(
        torch.float32)


def from_targets(t: torch.Tensor, scale: float, n_wl: int) -> torch.Tensor:
    """Inverse of :func:`to_targets`."""
    n, P, _ = t.shape
    r = t.to(torch.float64).reshape(n, P, n_wl, 2).permute(0, 2, 1, 3) * scale
    return torch.view_as_complex(r.contiguous())


def label_scale(labels: torch.Tensor) -> float:
    return float(torch.sqrt((labels.abs() ** 2).mean()))


def _real_view(x: torch.Tensor) -> torch.Tensor:
    return torch.view_as_real(x) if x.is_complex() else x


def rel_l2_per_sample(pred: torch.Tensor, true: torch.Tensor) -> torch.Tensor:
    """||pred - true|| / ||true|| per sample (complex values count re and im)."""
    d = _real_view(pred - true).reshape(pred.shape[0], -1).to(torch.float64)
    t = _real_view(true).reshape(true.shape[0], -1).to(torch.float64)
    return d.norm(dim=1) / t.norm(dim=1).clamp_min(1e-300)


def make_dataset(n: int, seed: int, labeler: FDTDLabeler, sigma_range=(2.0, 6.0)):
    """(design eps float32 (n, 128, 128) on the labeler's device, complex labels)."""
    masks, _ = blob_designs(n, seed, sigma_range, labeler.setup.design, labeler.device)
    eps = design_eps(masks)
    return eps, labeler.label(eps)


def cell_steps(n: int, setup: TMzSetup = TMzSetup()) -> int:
    return n * setup.side * setup.side * setup.n_steps


__all__: Sequence[str] = ["TMzSetup", "blob_designs", "design_eps", "FDTDLabeler", "to_targets",
                          "from_targets", "label_scale", "rel_l2_per_sample", "make_dataset",
                          "cell_steps"]
