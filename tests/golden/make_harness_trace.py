"""Record how DiffNano's own benchmark harness drives an FDTD solver class.

Run once, in a container that has the reference checkout (read-only); its
location comes from ``DIFFNANO_REFERENCE`` (default ``/root/reference``)::

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_harness_trace.py

It runs the reference's unmodified harness on the CPU --
``FDTDBenchmarkSuite().run(cls, BenchmarkConfig(...))``
(``diffnano/solvers/fdtd_benchmark.py:96-204``) and
``SystolicUpdateEvaluator().measure_bandwidth(solver, grid)`` (``:313-391``)
-- with ``cls`` a recording subclass of the reference's own
``FDTDSolver3D``.  The subclass logs every constructor call (keyword
arguments), every ``forward`` (the geometry's shape, dtype and
``requires_grad``) and every ``_time_step`` call (argument shapes and
dtypes), and keeps the eps tensors the harness built so their gradients can
be stored after the harness has called ``backward`` on them.

Outputs, read by ``tests/test_harness.py`` on the GPU box (where the
reference does not exist): ``harness_trace.json`` (the call log and the
harness's result records) and ``harness_trace.npz`` (per backward mode: the
eps the harness passed, the reference's field and eps.grad).
"""

from __future__ import annotations

import dataclasses
import json
import os
import sys

import numpy as np
import torch

REF = os.environ.get("DIFFNANO_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REF)

from diffnano.solvers.fdtd3d import FDTDSolver3D  # noqa: E402  (reference)
from diffnano.solvers.fdtd_benchmark import (  # noqa: E402  (reference)
    BenchmarkConfig,
    FDTDBenchmarkSuite,
    SystolicUpdateEvaluator,
)

GRID = (16, 16, 16)
N_STEPS = 40
EVENTS: list = []
KEPT: list = []


def _describe(t):
    if isinstance(t, torch.Tensor):
        return {"shape": list(t.shape), "dtype": str(t.dtype), "device": t.device.type,
                "requires_grad": bool(t.requires_grad)}
    return repr(t)


def _from_harness() -> bool:
    """True when the logged method was called from the harness file itself
    (the reference solver also calls its own ``_time_step`` internally)."""
    return sys._getframe(2).f_code.co_filename.endswith("fdtd_benchmark.py")


class RecordingSolver(FDTDSolver3D):
    """The reference solver with every call the harness makes logged."""

    def __init__(self, **kw):
        EVENTS.append({"call": "__init__", "kwargs": {k: (list(v) if isinstance(v, tuple) else v)
                                                     for k, v in kw.items()}})
        super().__init__(**kw)

    def forward(self, geometry, wavelengths=None, *, source=None):
        EVENTS.append({"call": "forward", "geometry": _describe(geometry),
                       "wavelengths": wavelengths, "source": source})
        r = super().forward(geometry, wavelengths, source=source)
        KEPT.append((geometry, r.field.detach().clone()))
        return r

    def _time_step(self, *args):
        if _from_harness():
            EVENTS.append({"call": "_time_step", "args": [_describe(a) for a in args]})
        return super()._time_step(*args)


def main() -> None:
    torch.set_num_threads(os.cpu_count() or 1)
    cfg = BenchmarkConfig(grid_sizes=[GRID], n_time_steps=N_STEPS, device="cpu")
    results = FDTDBenchmarkSuite().run(RecordingSolver, cfg)
    arrays = {}
    for mode, (eps, field) in zip(cfg.backward_modes, KEPT):
        arrays[f"eps_{mode}"] = eps.detach().numpy()
        arrays[f"field_{mode}"] = field.numpy()
        arrays[f"grad_{mode}"] = eps.grad.numpy()
    n_fwd = len(EVENTS)
    solver = RecordingSolver(grid_shape=GRID, dl=20.0, wavelength_nm=1550.0, pml_layers=0,
                             n_steps=N_STEPS, device="cpu", courant=0.35)
    bw = SystolicUpdateEvaluator().measure_bandwidth(solver, GRID)
    trace = {"harness": "diffnano/solvers/fdtd_benchmark.py",
             "config": dataclasses.asdict(cfg),
             "suite_events": EVENTS[:n_fwd],
             "bandwidth_events": EVENTS[n_fwd:],
             "suite_results": [dataclasses.asdict(r) for r in results],
             "bandwidth_result_keys": sorted(bw)}
    with open(os.path.join(HERE, "harness_trace.json"), "w") as fh:
        json.dump(trace, fh, indent=1, default=list)
    np.savez_compressed(os.path.join(HERE, "harness_trace.npz"), **arrays)
    print(f"{len(EVENTS)} calls recorded; results: "
          + "; ".join(f"{r.backward_mode} cos={r.gradient_cosine_vs_autograd}" for r in results))


if __name__ == "__main__":
    main()
