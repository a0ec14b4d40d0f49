"""diffnano_b200 -- B200-native (sm_100a) differentiable Yee FDTD.

Drop-in for DiffNano's FDTD solvers (``diffnano.FDTDSolver2D`` /
``diffnano.FDTDSolver3D``): same constructors, ``forward`` and
``time_series``, computed by hand-written CUDA kernels in
``_native/libdn_fdtd.so`` (C ABI: ``include/dn_fdtd.h``).
"""

from __future__ import annotations

__version__ = "0.1.0"

__all__ = ["FDTDSolver2D", "FDTDSolver3D", "SimResult", "Solver"]


def __getattr__(name):
    if name in ("FDTDSolver2D", "FDTDSolver3D", "SimResult", "Solver"):
        from diffnano_b200 import solvers

        return getattr(solvers, name)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
