"""B200 3-D FDTD solver, drop-in for ``diffnano.solvers.fdtd3d.FDTDSolver3D``.

Same constructor, attributes, ``forward`` and ``time_series`` as the
reference (``diffnano/solvers/fdtd3d.py:222-700``); every time step runs in
the fused ``dn_fdtd3d_run`` CUDA kernel (``include/dn_fdtd.h``).  Additions,
all optional keyword arguments: ``dtype`` (torch.float32 default,
torch.float64 for validation), DFT ``monitors``, ``cpml_axes``
("reference" = the reference's coefficient broadcasting, cubic grids only;
"physical" = every profile along its own axis, any grid) and
``source["component"]`` ("Ex"/"Ey"/"Ez", default "Ez" as in the reference).
"""

from __future__ import annotations

import math
from collections.abc import Sequence

import torch

from diffnano_b200 import _lib
from diffnano_b200.solvers import _setup
from diffnano_b200.solvers._common import (
    GridShapeError,
    as_wavelength_tensor,
    monitor_metadata,
    parse_monitors,
)
from diffnano_b200.solvers._engine import Engine, compute_device, to_result_device
from diffnano_b200.solvers._result import SimResult

__all__ = ["FDTDSolver3D"]

_FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
_OUT = ("Ez", "Ex", "Ey")  # field order of SimResult.field (fdtd3d.py:639)


class FDTDSolver3D:
    """Differentiable 3-D FDTD solver (all six components).

    Parameters are the reference's (``fdtd3d.py:250-262``) plus keyword-only
    ``dtype``, ``monitors`` and ``cpml_axes``.  ``backward`` accepts the
    reference's values: "auto" (and any other string), "checkpoint",
    "time_reversal".  ``device`` is where inputs and results live; the
    kernels always run on a CUDA device.
    """

    def __init__(self, grid_shape: tuple[int, int, int] = (30, 30, 30), dl: float = 20.0,
                 wavelength_nm: float = 1550.0, pml_layers: int = 5, n_steps: int = 500,
                 courant: float = 0.4, device: str | torch.device = "cpu",
                 use_checkpoint: bool = False, checkpoint_segments: int = 4,
                 backward: str = "auto", *, dtype: torch.dtype = torch.float32, monitors=None,
                 cpml_axes: str = "reference"):
        self.grid_shape = grid_shape
        self.dl = dl
        self.wavelength_nm = wavelength_nm
        self.pml_layers = pml_layers
        self.n_steps = n_steps
        self.courant = courant
        self._device = torch.device(device)
        self.use_checkpoint = use_checkpoint
        self.checkpoint_segments = checkpoint_segments
        self.backward = backward
        self.dtype = dtype
        self.monitors = monitors
        if cpml_axes not in ("reference", "physical"):
            raise ValueError(f"cpml_axes must be 'reference' or 'physical', got {cpml_axes!r}")
        self.cpml_axes = cpml_axes
        self.dt = courant * dl / math.sqrt(3.0)
        self.omega = 2 * math.pi / wavelength_nm

    @property
    def device(self) -> torch.device:
        return self._device

    # ------------------------------------------------------------------
    def _axes(self) -> int:
        D, H, W = self.grid_shape
        if self.cpml_axes == "reference":
            if not (D == H == W):
                raise GridShapeError(
                    f"grid {tuple(self.grid_shape)} is not cubic: the reference's CPML "
                    "broadcasting (fdtd3d.py:402-463) only exists for cubic grids; "
                    "use cpml_axes='physical'")
            return _lib.DN_AXES_REFERENCE
        return _lib.DN_AXES_PHYSICAL

    def _prep_eps(self, geometry: torch.Tensor) -> torch.Tensor:
        eps = geometry
        if eps.dim() == 4:
            eps = eps.squeeze(0)
        if eps.dim() == 2:
            eps = eps.unsqueeze(0)
        if tuple(eps.shape) != tuple(self.grid_shape):
            raise GridShapeError(f"geometry shape {tuple(geometry.shape)} does not match "
                                 f"grid_shape {tuple(self.grid_shape)}")
        return eps

    def _make_engine(self, n_steps: int, source: dict, monitors, probe=None) -> Engine:
        shape = tuple(self.grid_shape)
        axes = self._axes()
        comp = _setup.component_id(source.get("component", "Ez"), ("Ex", "Ey", "Ez"))
        box = _setup.source_box_3d(shape, source)
        wave = _setup.waveform_table(n_steps, self.dt, self.omega, source)
        specs = parse_monitors(monitors, shape, True, self.wavelength_nm, "Ez", _FIELDS)
        pr = None
        if probe is not None:
            pos = tuple(int(v) for v in probe)
            if not all(0 <= p < n for p, n in zip(pos, shape)):
                raise ValueError(f"probe {pos} outside the grid {shape}")
            pr = (_lib.DN_EZ, pos)
        return Engine(is3d=True, shape=shape, dl=self.dl, dt=self.dt, pml_layers=self.pml_layers,
                      dtype=self.dtype, device=compute_device(self._device), n_steps=n_steps,
                      wave=wave, src_box=box, src_comp=comp, monitors=specs, probe=pr, axes=axes)

    # ------------------------------------------------------------------
    def forward(self, geometry: torch.Tensor,
                wavelengths: Sequence[float] | torch.Tensor | None = None, *,
                source: dict | None = None, monitors=None) -> SimResult:
        """Run the 3-D simulation (``fdtd3d.py:564-650``).

        ``field`` is ``stack([Ez, Ex, Ey])``, shape ``(3, D, H, W)``, in the
        solver's ``dtype`` on ``device``.  ``monitors`` (here or at
        construction) adds ``metadata["monitors"]``.
        """
        wl = as_wavelength_tensor(wavelengths, self.wavelength_nm, self._device)
        src = source or {"type": "gaussian_pulse"}
        eps = self._prep_eps(geometry)
        mons = monitors if monitors is not None else self.monitors
        eng = self._make_engine(self.n_steps, src, mons)
        from diffnano_b200.solvers._adjoint import run_forward

        field, dfts = run_forward(self, eng, eps, _OUT)
        meta = {"n_steps": self.n_steps, "dt": self.dt, "courant": self.courant,
                "grid_shape": self.grid_shape}
        if self.backward == "time_reversal":
            meta["backward"] = "time_reversal"
        if eng.monitors:
            meta["monitors"] = monitor_metadata(
                eng, [to_result_device(d, self._device) for d in dfts])
        return SimResult(field=to_result_device(field, self._device), wavelengths=wl,
                         metadata=meta)

    def time_series(self, eps_r: torch.Tensor, probe: tuple[int, int, int],
                    source: dict | None = None, n_steps: int | None = None) -> torch.Tensor:
        """Ez at ``probe`` after every step, shape ``(n_steps,)``
        (``fdtd3d.py:652-700``)."""
        src = source or {"type": "gaussian_pulse"}
        eps = self._prep_eps(eps_r)
        steps = n_steps or self.n_steps
        eng = self._make_engine(steps, src, (), probe)
        with torch.no_grad():
            eng.set_eps(eps)
            eng.run(0, steps)
        eng.check_status()
        return eng.probe_out.to(self._device)

    # ------------------------------------------------------------------
    # reference-compatible private hooks
    # ------------------------------------------------------------------
    def _source_waveform(self, step: int, source: dict) -> torch.Tensor:
        """FP64 scalar tensor of the source amplitude at ``step``."""
        w = _setup.waveform_table(step + 1, self.dt, self.omega, source)[step]
        return w.to(self._device)

    def _build_source_mask(self, source: dict) -> torch.Tensor:
        """Dense FP64 ``(D, H, W)`` 0/1 mask of the injected cells."""
        m = torch.zeros(*self.grid_shape, dtype=torch.float64, device=self._device)
        box = _setup.source_box_3d(tuple(self.grid_shape), source)
        if box is not None:
            m[tuple(slice(a, b) for a, b in box)] = 1.0
        return m

    def _time_step(self, Ex, Ey, Ez, Hx, Hy, Hz, eps_r, mu_r):
        """One step without source (``fdtd3d.py:378-465``), the hook the
        reference's bandwidth harness times (``fdtd_benchmark.py:346-363``);
        mu_r must be 1.  Runs the fused kernel in the inputs' dtype (float32
        or float64) straight from the caller's tensors when they allow it; the
        set-up is cached across calls (``_stephook.StepHook``)."""
        from diffnano_b200.solvers._stephook import hook_for

        dtype = Ex.dtype if Ex.dtype in (torch.float32, torch.float64) else self.dtype
        h = hook_for(self, True, dtype, compute_device(Ex.device), axes=self._axes())
        return h.step((Ex, Ey, Ez, Hx, Hy, Hz), eps_r, mu_r)
