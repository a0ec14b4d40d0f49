"""Batched 2-D instances against the CPU FP64 oracle directly.

A small ragged batch in the shape of the batched workload: square sides
48-160, blob designs with -1 / 0 / +1-cell erosion / dilation variants
(``-max_pool2d(-x, 3, 1, 1)`` / ``max_pool2d(x, 3, 1, 1)``,
``diffnano/design/constraints_shared/primitives.py:56-60``), eight source
wavelengths in 1450-1650 nm, step counts that grow with the side, a DFT row
monitor per instance.  Every instance's final Ez, monitor DFT and dL/deps
(L = sum of a seeded weighting of the field plus sum |DFT|^2) are compared
with ``oracle.fdtd_ref.run_2d`` and its autograd -- for the thread-block
cluster kernel (gradient-free), the persistent kernel (gradient-free and with
gradients) in FP32 (relative L2 1e-5) and FP64 (1e-12; gradients 1e-9).
"""

from __future__ import annotations

import math

import pytest
import torch
from conftest import rel_l2

from diffnano_b200.solvers.batch2d import BatchInstance, FDTDBatch2D
from diffnano_b200.workloads import blob_eps_2d, gaussian_pulse_for_band
from oracle import fdtd_ref as R

pytestmark = pytest.mark.gpu

SIDES = [48, 64, 96, 128, 160, 64, 96, 48]
WLS = torch.linspace(1450.0, 1650.0, 8).tolist()
TOL = {torch.float32: (1e-5, 1e-5, 1e-4), torch.float64: (1e-12, 1e-12, 1e-9)}


def _batch():
    specs, eps = [], []
    for n, side in enumerate(SIDES):
        T = 200 + side  # more steps on larger grids
        src = gaussian_pulse_for_band(WLS[n], 200.0)
        src.update(row=12, spread=350.0, t0=1050.0)
        # the monitor row is close enough to the source row for the pulse
        # (peak at step ~150, ~0.35 cells per step) to cross it well within T
        mon_row = min(side - 12, 40)
        specs.append(BatchInstance(grid_shape=(side, side), n_steps=T, dl=20.0,
                                   wavelength_nm=WLS[n], pml_layers=10, courant=0.5, source=src,
                                   monitor={"row": mon_row, "wavelengths_nm": [WLS[n], 1550.0]}))
        eps.append(blob_eps_2d(side, side // 2, seed=n // 3, sigma_cells=2.0,
                               variant=(n % 3) - 1))
    return specs, eps


def _weights(specs):
    g = torch.Generator().manual_seed(77)
    return [torch.randn(*s.grid_shape, dtype=torch.float64, generator=g) for s in specs]


def _oracle(spec, eps, grad):
    e = eps.clone().requires_grad_(grad)
    H, W = spec.grid_shape
    r = spec.monitor["row"]
    o = R.run_2d(e, dl=spec.dl, dt=spec.dt, omega=spec.omega, pml_layers=spec.pml_layers,
                 n_steps=spec.n_steps, source=spec.source,
                 monitors=[{"component": "Ez", "box": ((r, r + 1), (0, W)),
                            "wavelengths_nm": spec.monitor["wavelengths_nm"]}])
    return e, o["Ez"], o["monitors"][0]


def _loss(field, dft_ri, w):
    return (field * w).sum() + (dft_ri ** 2).sum()


@pytest.fixture(scope="module")
def reference():
    specs, eps = _batch()
    w = _weights(specs)
    torch.set_num_threads(max(1, torch.get_num_threads()))
    out = []
    for spec, e, wi in zip(specs, eps, w):
        ee, f, d = _oracle(spec, e, True)
        _loss(f, d, wi).backward()
        out.append((f.detach(), d.detach(), ee.grad))
    return specs, eps, w, out


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("cluster", [None, False])
def test_batched_forward_vs_oracle(cuda, reference, dtype, cluster):
    specs, eps, _, ref = reference
    b = FDTDBatch2D(specs, "TM", dtype, cuda, cluster=cluster)
    with torch.no_grad():
        fields, dfts = b.forward([e.to(cuda) for e in eps])
    b._build(False)
    assert b.uses_cluster(False) == (cluster is None)
    tf, td, _ = TOL[dtype]
    for n, (f, d, (rf, rd, _)) in enumerate(zip(fields, dfts, ref)):
        assert rel_l2(f, rf) < tf, (n, rel_l2(f, rf))
        got = torch.view_as_real(d.to(torch.complex128)).reshape(rd.shape)
        assert rel_l2(got, rd) < td, (n, rel_l2(got, rd))


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_batched_gradients_vs_oracle(cuda, reference, dtype):
    specs, eps, w, ref = reference
    b = FDTDBatch2D(specs, "TM", dtype, cuda, checkpoint_interval=int(math.sqrt(200)))
    e_dev = [e.to(cuda).requires_grad_(True) for e in eps]
    fields, dfts = b.forward(e_dev)
    loss = sum(_loss(f.double(), torch.view_as_real(d.to(torch.complex128)), wi.to(cuda))
               for f, d, wi in zip(fields, dfts, w))
    loss.backward()
    tf, td, tg = TOL[dtype]
    for n, (f, e, (rf, _, rg)) in enumerate(zip(fields, e_dev, ref)):
        assert rel_l2(f, rf) < tf
        assert rel_l2(e.grad, rg) < tg, (n, rel_l2(e.grad, rg))
