"""Serve the B200 solvers under DiffNano's own module paths.

Most of DiffNano's callers take the solver class as an argument
(``FDTDBenchmarkSuite.run(fdtd3d_class, cfg)``,
``diffnano/solvers/fdtd_benchmark.py:96-133``) and need nothing from here.
Others import it by module path inside their methods --
``from diffnano.solvers.fdtd3d import FDTDSolver3D`` in ``FDTDGPUBenchmark``,
``FDTDXCrossValidator`` and ``MultiScaleMetalens``
(``diffnano/solvers/fdtd_benchmark_gpu.py:225,443,476,688,811``).
:func:`install` makes those paths resolve to this package's solvers:

* ``sys.modules["diffnano.solvers.fdtd3d"]`` / ``["diffnano.solvers.fdtd2d"]``
  become :mod:`diffnano_b200.solvers.fdtd3d` / ``fdtd2d``; an import by that
  path is answered from ``sys.modules`` before any file is searched, so it
  works whether or not DiffNano itself is installed;
* if ``diffnano.solvers`` is already imported, its ``fdtd3d`` / ``fdtd2d``
  submodule attributes and its re-exported ``FDTDSolver3D`` /
  ``FDTDSolver2D`` names are pointed at the drop-ins too (it bound the
  originals when it was first imported).

Call it before the callers run; :func:`uninstall` restores what was there.
"""

from __future__ import annotations

import sys

_SAVED: dict = {}
_NAMES = {"fdtd3d": "FDTDSolver3D", "fdtd2d": "FDTDSolver2D"}


def install() -> None:
    """Point DiffNano's FDTD module paths at the B200 drop-ins."""
    from diffnano_b200.solvers import fdtd2d, fdtd3d

    mods = {"fdtd3d": fdtd3d, "fdtd2d": fdtd2d}
    pkg = sys.modules.get("diffnano.solvers")
    for sub, mod in mods.items():
        key = f"diffnano.solvers.{sub}"
        if key not in _SAVED:
            _SAVED[key] = sys.modules.get(key)
        sys.modules[key] = mod
        if pkg is not None:
            for attr, val in ((sub, mod), (_NAMES[sub], getattr(mod, _NAMES[sub]))):
                _SAVED.setdefault(("attr", attr), getattr(pkg, attr, None))
                setattr(pkg, attr, val)


def uninstall() -> None:
    """Undo :func:`install`."""
    pkg = sys.modules.get("diffnano.solvers")
    for key, val in list(_SAVED.items()):
        if isinstance(key, tuple):
            if pkg is not None:
                if val is None:
                    if hasattr(pkg, key[1]):
                        delattr(pkg, key[1])
                else:
                    setattr(pkg, key[1], val)
        elif val is None:
            sys.modules.pop(key, None)
        else:
            sys.modules[key] = val
    _SAVED.clear()
