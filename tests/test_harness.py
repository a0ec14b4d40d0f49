"""DiffNano's benchmark harness driving the drop-in solver.

``tests/golden/harness_trace.json`` / ``.npz`` record what the reference's own
harness does with a solver class (``make_harness_trace.py`` ran
``FDTDBenchmarkSuite().run`` and ``SystolicUpdateEvaluator().measure_bandwidth``
from ``diffnano/solvers/fdtd_benchmark.py`` with a logging subclass of the
reference solver): the constructor keywords (``pml_layers=0``,
``courant=0.35``, the three backward modes), the eps tensors it passed, the
reference's fields and gradients, and the ``_time_step`` calls of the
bandwidth probe.  The GPU tests replay that call sequence on the B200 solver
(the reference is not present on the GPU machine) and check the results the
harness would compute; the CPU tests cover :mod:`diffnano_b200.compat`, which
lets callers that import the solver by DiffNano's module path
(``fdtd_benchmark_gpu.py:225,443,476,688,811``) reach the drop-in.
"""

from __future__ import annotations

import json
import math
import os
import sys
import time

import numpy as np
import pytest
import torch
from conftest import GOLDEN, rel_l2

import diffnano_b200 as dn
from diffnano_b200 import compat
from oracle import fdtd_ref as R

TRACE = json.load(open(os.path.join(GOLDEN, "harness_trace.json")))
ARR = dict(np.load(os.path.join(GOLDEN, "harness_trace.npz")))


def _cos(a, b):
    a, b = a.double().flatten().cpu(), b.double().flatten().cpu()
    return float(a @ b / (a.norm() * b.norm()))


# ---------------------------------------------------------------------------
# CPU: module-path aliasing
# ---------------------------------------------------------------------------
def _fake_reference(tmp_path):
    """A package laid out like DiffNano's solvers: the package re-exports the
    class from its submodule, and a harness module imports it lazily."""
    pkg = tmp_path / "diffnano" / "solvers"
    pkg.mkdir(parents=True)
    (tmp_path / "diffnano" / "__init__.py").write_text("")
    (pkg / "__init__.py").write_text("from diffnano.solvers.fdtd3d import FDTDSolver3D\n")
    (pkg / "fdtd3d.py").write_text("class FDTDSolver3D:\n    origin = 'reference'\n")
    (pkg / "fdtd2d.py").write_text("class FDTDSolver2D:\n    origin = 'reference'\n")
    (pkg / "harness.py").write_text(
        "def solver_class():\n"
        "    from diffnano.solvers.fdtd3d import FDTDSolver3D\n"
        "    return FDTDSolver3D\n")
    return str(tmp_path)


@pytest.fixture
def clean_modules(monkeypatch):
    saved = {k: v for k, v in sys.modules.items() if k == "diffnano" or k.startswith("diffnano.")}
    yield
    compat.uninstall()
    for k in [k for k in sys.modules if k == "diffnano" or k.startswith("diffnano.")]:
        del sys.modules[k]
    sys.modules.update(saved)


@pytest.mark.parametrize("order", ["install_first", "import_first"])
def test_compat_install_reaches_the_drop_in(tmp_path, monkeypatch, clean_modules, order):
    monkeypatch.syspath_prepend(_fake_reference(tmp_path))
    if order == "import_first":
        import diffnano.solvers  # noqa: F401  (binds the original class first)

        compat.install()
    else:
        compat.install()
        import diffnano.solvers  # noqa: F401
    import diffnano.solvers.harness as h

    assert h.solver_class() is dn.FDTDSolver3D
    assert sys.modules["diffnano.solvers"].FDTDSolver3D is dn.FDTDSolver3D
    from diffnano.solvers.fdtd2d import FDTDSolver2D

    assert FDTDSolver2D is dn.FDTDSolver2D
    compat.uninstall()
    if order == "import_first":
        assert sys.modules["diffnano.solvers"].FDTDSolver3D.origin == "reference"
    assert "diffnano.solvers.fdtd3d" not in sys.modules or \
        sys.modules["diffnano.solvers.fdtd3d"] is not dn.solvers.fdtd3d


def test_trace_records_the_reference_harness_calls():
    """The recorded call sequence is the harness's (no solver internals)."""
    ev = TRACE["suite_events"]
    assert [e["call"] for e in ev] == ["__init__", "forward"] * 3
    modes = []
    for e in ev[::2]:
        kw = e["kwargs"]
        assert kw["pml_layers"] == 0 and kw["courant"] == 0.35 and kw["dl"] == 20.0
        modes.append("time_reversal" if kw.get("backward") == "time_reversal" else
                     "checkpoint" if kw.get("use_checkpoint") else "autograd")
    assert modes == TRACE["config"]["backward_modes"]
    bw = TRACE["bandwidth_events"]
    assert sum(e["call"] == "_time_step" for e in bw) == 7  # 2 warm-up + 5 timed
    assert all(len(e["args"]) == 8 for e in bw if e["call"] == "_time_step")


# ---------------------------------------------------------------------------
# GPU: replay of the harness on the drop-in
# ---------------------------------------------------------------------------
@pytest.mark.gpu
def test_benchmark_suite_sequence_on_the_drop_in(cuda):
    """``FDTDBenchmarkSuite.run`` with device="cuda": each mode's solver is
    built with the harness's keywords, eps.grad comes from
    ``result.field.sum().backward()``; fields and gradients match the
    reference's (FP32 kernels: 1e-5 / 1e-4) and the modes agree (the
    harness's cosine-vs-autograd column)."""
    ev = TRACE["suite_events"]
    grads = {}
    for init, fwd, mode in zip(ev[::2], ev[1::2], TRACE["config"]["backward_modes"]):
        kw = dict(init["kwargs"], device="cuda")
        kw["grid_shape"] = tuple(kw["grid_shape"])
        s = dn.FDTDSolver3D(**kw)
        eps = torch.tensor(ARR[f"eps_{mode}"]).to(cuda).requires_grad_(True)
        assert list(eps.shape) == fwd["geometry"]["shape"]
        torch.cuda.reset_peak_memory_stats()
        r = s.forward(eps)
        r.field.sum().backward()
        assert eps.grad is not None
        assert rel_l2(r.field, ARR[f"field_{mode}"]) < 1e-5, mode
        assert rel_l2(eps.grad, ARR[f"grad_{mode}"]) < 1e-4, mode
        grads[mode] = eps.grad.detach().clone()
    for mode in ("time_reversal", "checkpoint"):
        assert _cos(grads[mode], grads["autograd"]) > 0.999999


@pytest.mark.gpu
def test_bandwidth_probe_sequence_on_the_drop_in(cuda):
    """``SystolicUpdateEvaluator.measure_bandwidth``'s seven ``_time_step``
    calls on FP64 device tensors (eps_r, mu_r = 1) advance the fields exactly
    like seven oracle steps."""
    init = TRACE["bandwidth_events"][0]["kwargs"]
    shape = tuple(init["grid_shape"])
    s = dn.FDTDSolver3D(**dict(init, grid_shape=shape, device="cuda"))
    assert str(s._device) == "cuda"
    g = torch.Generator().manual_seed(5)
    f = [torch.randn(*shape, dtype=torch.float64, generator=g) for _ in range(6)]
    eps = 1.5 + torch.rand(*shape, dtype=torch.float64, generator=g)
    mu = torch.ones(*shape, dtype=torch.float64)
    cur = [t.to(cuda) for t in f]
    calls = [e for e in TRACE["bandwidth_events"] if e["call"] == "_time_step"]
    ed, md = eps.to(cuda), mu.to(cuda)
    for _ in calls:
        cur = list(s._time_step(*cur, ed, md))
    torch.cuda.synchronize()
    n = shape[0]
    prof = (*R.cpml_profile(n, init["pml_layers"], init["dl"], s.dt),) * 3
    ref = f
    for _ in calls:
        ref = list(R.step_3d(*ref, eps, prof, s.dt, init["dl"]))
    for a, b in zip(cur, ref):
        assert rel_l2(a, b) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("W,dtype", [(13, torch.float64), (16, torch.float32),
                                     (18, torch.float32), (20, torch.float64)])
def test_time_step_hook_direct_and_padded_paths(cuda, W, dtype):
    """Direct path (rows a multiple of 16 bytes) and padded path (others),
    repeated calls on the cached set-up, host tensors, against the oracle."""
    shape = (12, 12, W) if W != 13 else (13, 13, 13)
    axes = "reference" if len(set(shape)) == 1 else "physical"
    s = dn.FDTDSolver3D(grid_shape=shape, pml_layers=3, device=cuda, cpml_axes=axes)
    g = torch.Generator().manual_seed(W)
    f = [torch.randn(*shape, dtype=torch.float64, generator=g) for _ in range(6)]
    eps = 1.5 + torch.rand(*shape, dtype=torch.float64, generator=g)
    prof = (*R.cpml_profile(shape[2], 3, 20.0, s.dt), *R.cpml_profile(shape[1], 3, 20.0, s.dt),
            *R.cpml_profile(shape[0], 3, 20.0, s.dt))
    ref = f
    for _ in range(3):
        ref = list(R.step_3d(*ref, eps, prof, s.dt, 20.0, axes=axes))
    tol = 1e-5 if dtype == torch.float32 else 1e-12
    for where in (cuda, "cpu"):
        cur = [t.to(where, dtype) for t in f]
        for _ in range(3):
            cur = list(s._time_step(*cur, eps.to(where), torch.ones_like(eps).to(where)))
        for a, b in zip(cur, ref):
            assert a.device.type == torch.device(where).type and a.dtype == dtype
            assert rel_l2(a, b) < tol
    with pytest.raises(ValueError):
        s._time_step(*[t.to(cuda, dtype) for t in f], eps.to(cuda),
                     torch.full_like(eps, 2.0).to(cuda))


@pytest.mark.gpu
def test_time_step_hook_costs_one_kernel_step(cuda):
    """The harness divides bytes by wall time around ``_time_step`` calls:
    at 256^3 FP64 a call through the hook takes the time of the kernel step
    itself (measured through the engine), within 25 %."""
    shape = (256, 256, 256)
    s = dn.FDTDSolver3D(grid_shape=shape, pml_layers=12, device=cuda, dtype=torch.float64)
    g = torch.Generator(device=cuda).manual_seed(0)
    f = [torch.randn(*shape, dtype=torch.float64, device=cuda, generator=g) for _ in range(6)]
    eps = 1.5 + torch.rand(*shape, dtype=torch.float64, device=cuda, generator=g)
    mu = torch.ones_like(eps)
    for _ in range(3):
        f = list(s._time_step(*f, eps, mu))
    torch.cuda.synchronize()
    n = 20
    t = time.perf_counter()
    for _ in range(n):
        f = list(s._time_step(*f, eps, mu))
    torch.cuda.synchronize()
    hook = (time.perf_counter() - t) / n
    eng = s._make_engine(n + 3, {"type": "gaussian_pulse"}, ())
    eng.set_eps(eps)
    eng.run(0, 3)
    torch.cuda.synchronize()
    t = time.perf_counter()
    eng.run(3, n)
    torch.cuda.synchronize()
    kern = (time.perf_counter() - t) / n
    gbs = 20 * 8 * math.prod(shape) / hook / 1e9  # the harness's byte count
    print(f"\n_time_step 256^3 FP64: {hook * 1e3:.3f} ms/call, kernel {kern * 1e3:.3f} ms/step, "
          f"harness figure {gbs:.0f} GB/s")
    assert hook < 1.25 * kern
