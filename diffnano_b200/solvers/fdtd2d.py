"""B200 2-D FDTD solver, drop-in for ``diffnano.solvers.fdtd2d.FDTDSolver2D``.

Same constructor, attributes, ``forward`` and ``time_series`` as the
reference (``diffnano/solvers/fdtd2d.py:91-524``); every time step runs in the
``dn_fdtd2d_run`` CUDA kernel (``include/dn_fdtd.h``).  Additions, all
optional keyword arguments: ``backward`` ("auto"/"autograd"/"time_reversal"/
"checkpoint"), ``dtype`` (torch.float32 default, torch.float64 for
validation), and DFT ``monitors``.
"""

from __future__ import annotations

import json
import math
from collections.abc import Sequence
from types import SimpleNamespace

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

__all__ = ["FDTDSolver2D"]

_TM_FIELDS = ("Ez", "Hx", "Hy")
_TE_FIELDS = ("Hz", "Ex", "Ey")


class FDTDSolver2D:
    """Differentiable 2-D FDTD solver (TM: Ez, Hx, Hy; TE: Hz, Ex, Ey).

    Parameters are the reference's (``fdtd2d.py:117-129``) plus keyword-only
    extensions ``backward``, ``dtype`` and ``monitors``.  ``device`` is where
    inputs and results live; the kernels always run on a CUDA device.
    """

    def __init__(self, grid_shape: tuple[int, int] = (100, 100), dl: float = 20.0,
                 wavelength_nm: float = 1550.0, polarization: str = "TM", pml_layers: int = 10,
                 n_steps: int = 1000, courant: float = 0.5, device: str | torch.device = "cpu",
                 use_checkpoint: bool = False, checkpoint_segments: int = 4, *,
                 backward: str = "auto", dtype: torch.dtype = torch.float32, monitors=None):
        self.grid_shape = grid_shape
        self.dl = dl
        self.wavelength_nm = wavelength_nm
        self.polarization = polarization.upper()
        if self.polarization not in ("TM", "TE"):
            raise ValueError(f"polarization must be 'TM' or 'TE', got {polarization!r}")
        self.pml_layers = pml_layers
        self.n_steps = n_steps
        self.courant = courant
        self._device = torch.device(device)
        self.use_checkpoint = use_checkpoint
        self.checkpoint_segments = checkpoint_segments
        self.backward = backward
        self.dtype = dtype
        self.monitors = monitors
        self.dt = courant * dl / math.sqrt(2.0)
        self.omega = 2 * math.pi / wavelength_nm

    @property
    def device(self) -> torch.device:
        return self._device

    # ------------------------------------------------------------------
    def _fields(self):
        return _TM_FIELDS if self.polarization == "TM" else _TE_FIELDS

    def _prep_eps(self, geometry: torch.Tensor) -> torch.Tensor:
        eps = geometry
        if eps.dim() == 3:
            eps = eps.squeeze(0)
        if tuple(eps.shape) != tuple(self.grid_shape):
            raise GridShapeError(f"geometry shape {tuple(geometry.shape)} does not match "
                                 f"grid_shape {tuple(self.grid_shape)}")
        return eps

    def _make_engine(self, n_steps: int, source: dict, monitors, probe=None) -> Engine:
        H, W = self.grid_shape
        inj = _lib.DN_EZ if self.polarization == "TM" else _lib.DN_HZ
        box = _setup.source_box_2d((H, W), source)
        wave = _setup.waveform_table(n_steps, self.dt, self.omega, source)
        specs = parse_monitors(monitors, (1, H, W), False, self.wavelength_nm, self._fields()[0],
                               self._fields())
        pr = None
        if probe is not None:
            y, x = int(probe[0]), int(probe[1])
            if not (0 <= y < H and 0 <= x < W):
                raise ValueError(f"probe {tuple(probe)} outside the grid {(H, W)}")
            pr = (inj, (0, y, x))
        return Engine(is3d=False, shape=(H, W), dl=self.dl, dt=self.dt,
                      pml_layers=self.pml_layers, dtype=self.dtype,
                      device=compute_device(self._device), n_steps=n_steps, wave=wave,
                      src_box=box, src_comp=inj, monitors=specs, probe=pr,
                      pol=_lib.DN_TM if self.polarization == "TM" else _lib.DN_TE)

    # ------------------------------------------------------------------
    def forward(self, geometry: torch.Tensor,
                wavelengths: Sequence[float] | torch.Tensor | None = None, *,
                source: dict | None = None, monitors=None) -> SimResult:
        """Run the 2-D simulation (``fdtd2d.py:412-484``).

        ``field`` is the final Ez (TM) or Hz (TE), shape ``(1, H, W)``, in
        the solver's ``dtype`` on ``device``.  ``source["probe"]=[y, x]``
        fills ``metadata["snapshots"]`` like the reference.  ``monitors``
        (here or at construction) adds ``metadata["monitors"]``.
        """
        wl = as_wavelength_tensor(wavelengths, self.wavelength_nm, self._device)
        src = source or {"type": "gaussian_pulse"}
        eps = self._prep_eps(geometry)
        mons = monitors if monitors is not None else self.monitors
        probe = src.get("probe", None)
        fast, eng, specs = None, None, None
        if probe is None and not (torch.is_grad_enabled() and eps.requires_grad):
            # the cluster-resident path needs only the parsed monitors, not a
            # per-step engine (field sets, tables and uploads on every call)
            H, W = self.grid_shape
            specs = parse_monitors(mons, (1, H, W), False, self.wavelength_nm,
                                   self._fields()[0], self._fields())
            fast = self._cluster_solve(eps, src, specs)
        if fast is not None:
            field, dfts = fast
        else:
            from diffnano_b200.solvers._adjoint import run_forward

            needs_grad = torch.is_grad_enabled() and eps.requires_grad
            eng = self._engine_for(src, mons, probe, reuse=not needs_grad)
            specs = eng.monitors
            field, dfts = run_forward(self, eng, eps, self._fields()[0])
        out_dev = self._device
        snapshots = []
        if probe is not None:
            snapshots = list(eng.probe_out.to(out_dev, copy=True).unbind(0))
        meta = {"polarization": self.polarization, "n_steps": self.n_steps, "dt": self.dt,
                "courant": self.courant, "snapshots": snapshots}
        if specs:
            meta["monitors"] = monitor_metadata(SimpleNamespace(monitors=specs),
                                                [to_result_device(d, out_dev) for d in dfts])
        return SimResult(field=to_result_device(field.unsqueeze(0), out_dev), wavelengths=wl,
                         metadata=meta)

    def _engine_for(self, src: dict, mons, probe, reuse: bool) -> Engine:
        """The per-step engine of a solve.  Gradient-free calls reuse one per
        set-up (every run resets its fields and writes eps, and the results
        are copies), which saves the field allocations and table uploads of a
        new engine; calls that autograd differentiates get a fresh one, since
        the backward pass replays from it.  Set-ups that are not plain JSON
        (tensors in the source or monitor dicts) are not cached."""
        if not reuse:
            return self._make_engine(self.n_steps, src, mons, probe)
        try:
            key = json.dumps([src, mons, probe, self.n_steps, str(self.dtype),
                              list(self.grid_shape), self.dl, self.wavelength_nm,
                              self.pml_layers, self.courant, self.polarization,
                              str(self._device)], sort_keys=True)
        except TypeError:
            return self._make_engine(self.n_steps, src, mons, probe)
        cache = self.__dict__.setdefault("_engine_cache", {})
        eng = cache.get(key)
        if eng is None:
            if len(cache) >= 4:
                cache.clear()
            eng = cache[key] = self._make_engine(self.n_steps, src, mons, probe)
        return eng

    def _cluster_solve(self, eps, src, specs):
        """Gradient-free solve with the whole grid in one thread-block cluster
        (``dn_batch2d_forward_cluster``) when the grid fits and there is at most
        one monitor (``specs``: the parsed monitors), on the injected field;
        None otherwise."""
        if len(specs) > 1:
            return None
        comp = _lib.DN_EZ if self.polarization == "TM" else _lib.DN_HZ
        mon = None
        if specs:
            m = specs[0]
            if m.component != comp:
                return None
            mon = {"box": [list(m.box[1]), list(m.box[2])], "wavelengths_nm": list(m.wavelengths)}
        key = json.dumps([src, mon, str(self.dtype), list(self.grid_shape), self.n_steps,
                          self.dl, self.wavelength_nm, self.pml_layers, self.courant,
                          self.polarization, str(self._device)], sort_keys=True, default=str)
        cache = self.__dict__.setdefault("_cluster_cache", {})
        if key not in cache:
            from diffnano_b200.solvers.batch2d import BatchInstance, FDTDBatch2D

            spec = BatchInstance(grid_shape=tuple(self.grid_shape), n_steps=self.n_steps,
                                 dl=self.dl, wavelength_nm=self.wavelength_nm,
                                 pml_layers=self.pml_layers, courant=self.courant,
                                 source={k: v for k, v in src.items() if k != "probe"},
                                 monitor=mon)
            b = FDTDBatch2D([spec], self.polarization, self.dtype,
                            compute_device(self._device), tile_rows=16)
            b._build(False)
            cache[key] = b if b.uses_cluster(False) else None
        b = cache[key]
        if b is None:
            return None
        with torch.no_grad():
            fields, dfts = b.run_forward([eps], grad=False)
        b.check_status()
        return fields[0], [d for d in dfts if d is not None]

    def time_series(self, eps_r: torch.Tensor, probe: tuple[int, int], source: dict | None = None,
                    n_steps: int | None = None) -> torch.Tensor:
        """Field at ``probe`` after every step, shape ``(n_steps,)``
        (``fdtd2d.py:486-524``; like the reference it stores ``probe`` into
        the caller's ``source`` dict)."""
        src = source or {"type": "gaussian_pulse"}
        src["probe"] = probe
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
        """Dense FP64 ``(H, W)`` 0/1 mask of the injected cells."""
        H, W = self.grid_shape
        m = torch.zeros(H, W, dtype=torch.float64, device=self._device)
        box = _setup.source_box_2d((H, W), source)
        if box is not None:
            m[box[1][0]:box[1][1], box[2][0]:box[2][1]] = 1.0
        return m

    def _single_step(self, fields: dict, eps_r: torch.Tensor, mu_r=None):
        """One source-free step through the cached per-step hook
        (``_stephook.StepHook``): the kernel runs straight from the caller's
        tensors when they are contiguous CUDA tensors of the compute dtype."""
        from diffnano_b200.solvers._stephook import hook_for

        first = fields[self._fields()[0]]
        dtype = first.dtype if first.dtype in (torch.float32, torch.float64) else self.dtype
        pol = _lib.DN_TM if self.polarization == "TM" else _lib.DN_TE
        h = hook_for(self, False, dtype, compute_device(first.device), pol=pol)
        return h.step(tuple(fields[n] for n in self._fields()), eps_r, mu_r)

    def _time_step_tm(self, Ez, Hx, Hy, eps_r, mu_r):
        """One TM step without source (``fdtd2d.py:233-267``); mu_r must be 1."""
        if self.polarization != "TM":
            raise ValueError("_time_step_tm on a TE solver")
        return self._single_step({"Ez": Ez, "Hx": Hx, "Hy": Hy}, eps_r, mu_r)

    def _time_step_te(self, Hz, Ex, Ey, eps_r, mu_r):
        """One TE step without source (``fdtd2d.py:269-303``); mu_r must be 1."""
        if self.polarization != "TE":
            raise ValueError("_time_step_te on a TM solver")
        return self._single_step({"Hz": Hz, "Ex": Ex, "Ey": Ey}, eps_r, mu_r)
