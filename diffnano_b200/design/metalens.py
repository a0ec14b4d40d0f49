"""The focusing problem of the 3-D inverse-design workload and its 2-D proxy.

3-D problem (the FDTD judges every design): a 384 x 384 x 192 grid (x, y, z;
arrays are (z, y, x)), dx = 25 nm, 12-cell CPML on every axis (``cpml_axes=
"physical"``), 3000 steps, Courant 0.4.  SiO2 (2.085) below z = 40, air above;
a design block z in [40, 80), x and y in [64, 320) (256 x 256 x 40 cells)
holds air/Si (1.0 / 12.1) mixtures.  An Ey-polarised Gaussian-pulse plane
wave (1.55 um centre, 0.2 um width) starts at z = 20 in the substrate; the
figure of merit is |DFT Ey(1.55 um)|^2 at the focal point (z = 150, y = x =
192), 1.75 um above the block.  The density is rho(z, x) in [0, 1] (40 x 256),
extruded along y inside the block (a cylindrical lens focusing in x); eps =
1 + 11.1 * tanh_projection(smooth_filter(rho, r = 4), beta, eta = 0.5).

2-D proxy (what the surrogate is trained on): the x-z cross-section through
the lens axis as a 2-D TMz grid (rows = z, 192; columns = x, 384) with the
same dx, time step, CPML depth, layers, source row and design region; 2-D Ez
plays the part of 3-D Ey.  The batched 2-D FDTD labels thousands of proxy
designs per launch with the DFT of Ez along the focal row.

Coarse 3-D model (:func:`coarse_model`, what the assisted loop proposes
with): the same lens on 2x larger cells, driven by the fine density.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, replace
from typing import Optional, Tuple

import torch

from ..solvers._fom import fom_abs2
from ..solvers.batch2d import BatchInstance, FDTDBatch2D
from ..solvers.fdtd3d import FDTDSolver3D
from ..workloads import EPS_AIR, EPS_SI, EPS_SIO2, gaussian_pulse_for_band
from .projection import density_to_eps


@dataclass(frozen=True)
class MetalensSetup:
    shape: Tuple[int, int, int] = (192, 384, 384)  # (z, y, x)
    dl: float = 25.0
    pml: int = 12
    courant: float = 0.4
    n_steps: int = 3000
    design_z: Tuple[int, int] = (40, 80)
    design_xy: Tuple[int, int] = (64, 320)
    src_z: int = 20
    focus_z: int = 150
    wavelengths_nm: Tuple[float, ...] = (1500.0, 1550.0, 1600.0)
    center_nm: float = 1550.0
    bandwidth_nm: float = 200.0
    eps_sub: float = EPS_SIO2
    eps_lo: float = EPS_AIR
    eps_hi: float = EPS_SI
    radius: float = 4.0
    eta: float = 0.5

    @property
    def design_shape(self) -> Tuple[int, int]:
        return (self.design_z[1] - self.design_z[0], self.design_xy[1] - self.design_xy[0])

    @property
    def dt(self) -> float:
        return self.courant * self.dl / math.sqrt(3.0)

    @property
    def focus_col(self) -> int:
        """Index of the focal point on the monitor line (the line spans the block in x)."""
        return self.shape[2] // 2 - self.design_xy[0]

    @property
    def center_index(self) -> int:
        return list(self.wavelengths_nm).index(self.center_nm)

    def cell_steps(self) -> int:
        D, H, W = self.shape
        return D * H * W * self.n_steps

    def scaled(self, s: int) -> "MetalensSetup":
        """The same layout on a grid ``s`` times smaller in every direction
        (same dx; for tests)."""
        D, H, W = self.shape
        f = lambda v: max(1, v // s)  # noqa: E731
        pml = max(6, self.pml // s)
        return replace(self, shape=(f(D), f(H), f(W)), n_steps=max(400, self.n_steps // s),
                       design_z=(f(self.design_z[0]), f(self.design_z[1])),
                       design_xy=(f(self.design_xy[0]), f(self.design_xy[1])),
                       src_z=max(f(self.src_z), pml + 2), focus_z=f(self.focus_z), pml=pml,
                       radius=max(1.0, self.radius / s))

    def coarsened(self, f: int) -> "MetalensSetup":
        """The same lens on cells ``f`` times larger: the same physical
        layout, source, focal point and simulated time (dt scales with dx),
        ``f``^4 times fewer cell-steps; the CPML keeps at least its physical
        depth in cells of the coarse grid (at least 3)."""
        D, H, W = self.shape
        if D % f or H % f or W % f:
            raise ValueError(f"grid {self.shape} is not divisible by {f}")
        g = lambda v: v // f  # noqa: E731
        return replace(self, shape=(g(D), g(H), g(W)), dl=self.dl * f,
                       n_steps=max(1, self.n_steps // f), pml=max(3, self.pml // f),
                       design_z=(g(self.design_z[0]), g(self.design_z[1])),
                       design_xy=(g(self.design_xy[0]), g(self.design_xy[1])),
                       src_z=g(self.src_z), focus_z=g(self.focus_z),
                       radius=self.radius / f)

    def eps_design(self, rho: torch.Tensor, beta: float) -> torch.Tensor:
        """(40, 256) density -> (40, 256) design-region eps (differentiable)."""
        return density_to_eps(rho, self.radius, beta, self.eta, "tanh", self.eps_lo, self.eps_hi)

    def source(self, is3d: bool) -> dict:
        src = gaussian_pulse_for_band(self.center_nm, self.bandwidth_nm)
        if is3d:
            src.update(plane="xy", z=self.src_z, component="Ey")
        else:
            src.update(row=self.src_z)
        return src


class Metalens3D:
    """FDTD evaluation of a density: FOM, its gradient (adjoint) and the focal-line DFT.

    ``design_map(rho, beta)`` gives the design block's (dz, dx) eps; by default
    the setup's own filter and projection.  :func:`coarse_model` passes the
    fine problem's map averaged over the coarse cells."""

    def __init__(self, setup: MetalensSetup = MetalensSetup(), device="cuda",
                 dtype=torch.float32, design_map=None):
        self.setup = s = setup
        self.design_map = design_map or s.eps_design
        self.device = torch.device(device)
        D, H, W = s.shape
        self.line_y = H // 2
        mon = {"component": "Ey", "box": ((s.focus_z, s.focus_z + 1), (H // 2, H // 2 + 1),
                                          (s.design_xy[0], s.design_xy[1])),
               "wavelengths_nm": list(s.wavelengths_nm)}
        self.solver = FDTDSolver3D(grid_shape=s.shape, dl=s.dl, wavelength_nm=s.center_nm,
                                   pml_layers=s.pml, n_steps=s.n_steps, courant=s.courant,
                                   device=self.device, backward="time_reversal", dtype=dtype,
                                   monitors=[mon], cpml_axes="physical")
        bg = torch.full(s.shape, s.eps_lo, dtype=torch.float32, device=self.device)
        bg[: s.design_z[0]] = s.eps_sub
        self.background = bg
        self.evaluations = 0

    def eps(self, rho: torch.Tensor, beta: float) -> torch.Tensor:
        s = self.setup
        e2 = self.design_map(rho, beta)  # (dz, dx)
        z0, z1 = s.design_z
        a, b = s.design_xy
        block = e2[:, None, :].expand(z1 - z0, b - a, b - a)
        eps = self.background.clone()
        eps[z0:z1, a:b, a:b] = block
        return eps

    def evaluate(self, rho: torch.Tensor, beta: float, grad: bool = True):
        """(fom, d fom / d rho or None, focal-line DFT complex (L, n_x))."""
        s = self.setup
        x = rho.detach().to(self.device, torch.float32).requires_grad_(grad)
        with torch.set_grad_enabled(grad):
            eps = self.eps(x, beta)
            r = self.solver.forward(eps, source=s.source(True))
            dft = r.metadata["monitors"][0]["dft"].reshape(len(s.wavelengths_nm), -1)
            fom = fom_abs2(dft[s.center_index, s.focus_col:s.focus_col + 1])
            if grad:
                fom.backward()
        self.evaluations += 1
        g = x.grad.detach() if grad else None
        return float(fom.detach()), g, dft.detach()

    def focal(self, rho: torch.Tensor, beta: float, c: complex = None, b: complex = 0j,
              grad: bool = False):
        """Complex focal-point DFT (centre wavelength) of ``rho``; with ``c``
        given, also the mapped intensity |c e + b|^2 and, with ``grad``, its
        gradient with respect to ``rho`` (the 3-D adjoint).  The interface of
        :meth:`Proxy2D.focal`."""
        s = self.setup
        x = rho.detach().to(self.device, torch.float32).clone().requires_grad_(grad)
        with torch.set_grad_enabled(grad):
            eps = self.eps(x, beta)
            r = self.solver.forward(eps, source=s.source(True))
            dft = r.metadata["monitors"][0]["dft"].reshape(len(s.wavelengths_nm), -1)
            e = dft[s.center_index, s.focus_col]
            self.evaluations += 1
            if c is None:
                return complex(e.detach()), None, None
            v = (c * e + b).abs() ** 2
            if grad:
                v.backward()
        return complex(e.detach()), float(v.detach()), (x.grad.detach() if grad else None)


def coarse_model(setup: MetalensSetup, factor: int = 2, device="cuda") -> Metalens3D:
    """The lens of ``setup`` on ``factor`` times coarser cells, driven by the
    fine density: the fine design eps (filter and projection on the fine
    grid) averaged over each coarse cell.  At factor 2 one forward + adjoint
    costs ~1/11 of the fine one."""
    cs = setup.coarsened(factor)

    def design_map(rho, beta):
        ef = setup.eps_design(rho, beta)
        return torch.nn.functional.avg_pool2d(ef[None, None], factor)[0, 0]

    return Metalens3D(cs, device, design_map=design_map)


class Proxy2D:
    """The 2-D cross-section of :class:`Metalens3D`, labelled by the batched FDTD."""

    def __init__(self, setup: MetalensSetup = MetalensSetup(), chunk: int = 2048,
                 device="cuda"):
        self.setup = setup
        self.chunk = chunk
        self.device = torch.device(device)
        D, _, W = setup.shape
        self.grid = (D, W)
        # the 3-D run's time step: Courant number of the 2-D grid
        self.courant2d = setup.dt * math.sqrt(2.0) / setup.dl
        self._batch: Optional[FDTDBatch2D] = None
        self._n = 0
        self.cell_steps = 0

    def instance(self) -> BatchInstance:
        s = self.setup
        return BatchInstance(grid_shape=self.grid, n_steps=s.n_steps, dl=s.dl,
                             wavelength_nm=s.center_nm, pml_layers=s.pml,
                             courant=self.courant2d, source=s.source(False),
                             monitor={"box": ((s.focus_z, s.focus_z + 1),
                                              (s.design_xy[0], s.design_xy[1])),
                                      "wavelengths_nm": list(s.wavelengths_nm)})

    def full_eps(self, eps_design: torch.Tensor) -> torch.Tensor:
        s = self.setup
        n = eps_design.shape[0]
        D, W = self.grid
        eps = torch.full((n, D, W), s.eps_lo, dtype=torch.float64, device=self.device)
        eps[:, : s.design_z[0]] = s.eps_sub
        eps[:, s.design_z[0]:s.design_z[1], s.design_xy[0]:s.design_xy[1]] = \
            eps_design.to(self.device, torch.float64)
        return eps

    def _solver2d(self):
        if getattr(self, "_s2d", None) is None:
            from ..solvers.fdtd2d import FDTDSolver2D

            s = self.setup
            D, W = self.grid
            self._s2d = FDTDSolver2D(grid_shape=(D, W), dl=s.dl, wavelength_nm=s.center_nm,
                                     polarization="TM", pml_layers=s.pml, n_steps=s.n_steps,
                                     courant=self.courant2d, device=self.device,
                                     dtype=torch.float32)
            fc = W // 2
            self._mon = [{"component": "Ez", "box": [[s.focus_z, s.focus_z + 1], [fc, fc + 1]],
                          "wavelengths_nm": [s.center_nm]}]
        return self._s2d

    def focal(self, rho: torch.Tensor, beta: float, c: complex = None, b: complex = 0j,
              grad: bool = False):
        """Complex focal-point DFT (centre wavelength) of the cross-section for
        density ``rho``, by one 2-D FDTD solve; with ``c`` given, also the
        mapped intensity |c e + b|^2 and, with ``grad``, its gradient with
        respect to ``rho`` (the 2-D adjoint kernels).  Returns (e, value,
        gradient or None)."""
        s = self.setup
        solver = self._solver2d()
        x = rho.detach().to(self.device, torch.float32).clone().requires_grad_(grad)
        with torch.set_grad_enabled(grad):
            eps = self.full_eps(s.eps_design(x, beta).unsqueeze(0))[0].to(torch.float32)
            r = solver.forward(eps, source=s.source(False), monitors=self._mon)
            e = r.metadata["monitors"][0]["dft"].reshape(-1)[0]
            self.cell_steps += self.grid[0] * self.grid[1] * s.n_steps * (3 if grad else 1)
            if c is None:
                return complex(e.detach()), None, None
            v = (c * e + b).abs() ** 2
            if grad:
                v.backward()
        return complex(e.detach()), float(v.detach()), (x.grad.detach() if grad else None)

    @torch.no_grad()
    def label(self, eps_design: torch.Tensor) -> torch.Tensor:
        """(n, 40, 256) design eps -> complex128 (n, L, 256) focal-row DFTs."""
        out = []
        for a in range(0, eps_design.shape[0], self.chunk):
            part = eps_design[a:a + self.chunk]
            n = part.shape[0]
            if self._batch is None or self._n != n:
                self._batch = FDTDBatch2D([self.instance() for _ in range(n)], "TM",
                                          torch.float32, self.device, tile_rows=16)
                self._n = n
            _, dfts = self._batch.run_forward(list(self.full_eps(part).unbind(0)))
            self._batch.check_status()
            out.append(torch.stack([d.reshape(d.shape[0], -1) for d in dfts]))
            self.cell_steps += n * self.grid[0] * self.grid[1] * self.setup.n_steps
        return torch.cat(out)


def random_densities(n: int, shape: Tuple[int, int], seed: int, device="cuda") -> torch.Tensor:
    """Seeded densities for the proxy's training set: 0.5 + a * (Gaussian-
    filtered unit noise), a ~ U(0, 0.8), clamped to [0, 1]; filter radius
    drawn from {2, 4, 8} cells.  Covers the near-uniform start of a design
    run as well as high-contrast layouts."""
    g = torch.Generator().manual_seed(seed)
    noise = torch.randn(n, *shape, generator=g)
    amp = torch.rand(n, 1, 1, generator=g) * 0.8
    radii = torch.tensor([2.0, 4.0, 8.0])[torch.randint(0, 3, (n,), generator=g)]
    noise = noise.to(device)
    out = torch.empty(n, *shape, device=device)
    from .projection import smooth_filter
    for r in radii.unique().tolist():
        sel = (radii == r).nonzero().flatten().to(device)
        f = smooth_filter(noise[sel], r)
        f = f / f.flatten(1).std(dim=1).clamp_min(1e-6)[:, None, None]
        out[sel] = f
    return (0.5 + amp.to(device) * out).clamp(0.0, 1.0)


def random_betas(n: int, seed: int, lo: float = 1.0, hi: float = 32.0,
                 levels: int = 16) -> torch.Tensor:
    """Projection sharpness per design, log-uniform on ``levels`` values."""
    g = torch.Generator().manual_seed(seed + 1)
    k = torch.randint(0, levels, (n,), generator=g).to(torch.float64)
    return lo * (hi / lo) ** (k / (levels - 1))


def proxy_dataset(proxy: Proxy2D, n: int, seed: int):
    """(design eps (n, 40, 256) float32, complex labels (n, L, 256))."""
    s = proxy.setup
    rho = random_densities(n, s.design_shape, seed, proxy.device)
    betas = random_betas(n, seed)
    eps = torch.empty_like(rho)
    for b in betas.unique().tolist():
        sel = (betas == b).nonzero().flatten().to(proxy.device)
        eps[sel] = s.eps_design(rho[sel], b)
    return eps, proxy.label(eps)
