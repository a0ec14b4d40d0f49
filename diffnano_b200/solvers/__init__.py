"""Solver interface and the B200 FDTD solvers.

Mirrors ``diffnano/solvers/__init__.py:47-81`` (the runtime-checkable
``Solver`` protocol) and its lazy exports of ``FDTDSolver2D`` and
``FDTDSolver3D``.
"""

from __future__ import annotations

from collections.abc import Sequence
from typing import Protocol, runtime_checkable

import torch

from diffnano_b200.solvers._result import SimResult

__all__ = ["Solver", "SimResult", "FDTDSolver2D", "FDTDSolver3D", "fom_abs2"]


@runtime_checkable
class Solver(Protocol):
    """Backend-agnostic forward-solver interface (``forward`` + ``device``)."""

    def forward(self, geometry: torch.Tensor,
                wavelengths: Sequence[float] | torch.Tensor | None, *,
                source: dict | None = None) -> SimResult: ...

    @property
    def device(self) -> torch.device: ...


def __getattr__(name):
    if name == "FDTDSolver2D":
        from diffnano_b200.solvers.fdtd2d import FDTDSolver2D

        return FDTDSolver2D
    if name == "FDTDSolver3D":
        from diffnano_b200.solvers.fdtd3d import FDTDSolver3D

        return FDTDSolver3D
    if name == "fom_abs2":
        from diffnano_b200.solvers._fom import fom_abs2

        return fom_abs2
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
