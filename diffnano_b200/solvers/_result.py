"""Simulation result container, same shape as DiffNano's ``SimResult``
(``diffnano/solvers/_result.py:8-35``): ``field``, ``wavelengths``,
``metadata`` and a ``device`` property."""

from __future__ import annotations

import torch


class SimResult:
    """Outputs of one simulation.

    Attributes
    ----------
    field : torch.Tensor
        Field data; ``(1, H, W)`` for the 2-D solver, ``(3, D, H, W)``
        (order Ez, Ex, Ey) for the 3-D solver.
    wavelengths : torch.Tensor
        Wavelengths in nm, ``(L,)``.
    metadata : dict
        Solver metadata (``n_steps``, ``dt``, ``courant``, ... and, when DFT
        monitors are requested, ``monitors``).
    """

    __slots__ = ("field", "wavelengths", "metadata")

    def __init__(self, field: torch.Tensor, wavelengths: torch.Tensor, metadata: dict | None = None):
        self.field = field
        self.wavelengths = wavelengths
        self.metadata = metadata or {}

    @property
    def device(self) -> torch.device:
        return self.field.device
