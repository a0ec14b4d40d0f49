"""Pieces shared by ``FDTDSolver2D`` and ``FDTDSolver3D``: argument
normalisation, monitor specs and the autograd wrapper around the kernels."""

from __future__ import annotations

import math

import torch

from diffnano_b200 import _lib
from diffnano_b200.solvers import _setup
from diffnano_b200.solvers._engine import MonitorSpec

F64 = torch.float64


class GridShapeError(ValueError, RuntimeError):
    """Grid/geometry shape mismatch (also a RuntimeError, which is what the
    reference's failed broadcasts raise)."""


def as_wavelength_tensor(wavelengths, default_nm: float, device) -> torch.Tensor:
    """``forward``'s ``wavelengths`` argument, normalised as the reference
    does (``fdtd2d.py:441-444``): metadata only."""
    if wavelengths is None:
        wavelengths = [default_nm]
    if not isinstance(wavelengths, torch.Tensor):
        wavelengths = torch.tensor(wavelengths, dtype=F64, device=device)
    return wavelengths


def parse_monitors(specs, shape3, is3d: bool, default_wl: float, default_comp: str,
                   allowed) -> list[MonitorSpec]:
    """Monitor dicts -> :class:`MonitorSpec` list (validated, ValueError)."""
    out = []
    for n, spec in enumerate(specs or ()):
        if not isinstance(spec, dict):
            raise ValueError(f"monitor spec must be a dict, got {type(spec).__name__}")
        comp = _setup.component_id(spec.get("component", default_comp), allowed)
        box = _setup.monitor_box(spec, shape3, is3d)
        wl = spec.get("wavelengths_nm", [default_wl])
        wl = [float(w) for w in (wl.tolist() if isinstance(wl, torch.Tensor) else wl)]
        if any(not (w > 0 and math.isfinite(w)) for w in wl):
            raise ValueError(f"monitor wavelengths must be positive: {wl}")
        out.append(MonitorSpec(name=str(spec.get("name", f"monitor{n}")), component=comp, box=box,
                               wavelengths=wl))
    if len(out) > _lib.DN_MAX_MONITORS:
        raise ValueError(f"at most {_lib.DN_MAX_MONITORS} monitors per solve")
    return out


def monitor_metadata(engine, dfts) -> list[dict]:
    """``metadata["monitors"]`` entries: name, component, box, wavelengths, dft."""
    names = {v: k for k, v in _lib.COMPONENTS.items()}
    return [dict(name=s.name, component=names[s.component], box=s.box,
                 wavelengths_nm=list(s.wavelengths), dft=d)
            for s, d in zip(engine.monitors, dfts)]


def checkpoint_interval(n_steps: int, use_checkpoint: bool, segments: int) -> int:
    """Steps between stored states for the adjoint sweep.

    With ``use_checkpoint`` the reference splits the run into
    ``checkpoint_segments`` segments (``fdtd2d.py:368``); otherwise the
    memory/recompute balance point sqrt(T) is used.
    """
    if use_checkpoint:
        return max(1, n_steps // max(1, segments))
    return max(1, int(math.ceil(math.sqrt(max(1, n_steps)))))
