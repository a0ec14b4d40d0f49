"""The FP32 3-D step runs two columns per lane by default; the one-column
kernel (``DN_FDTD3D_LANE_COLUMNS=1``, read once per process, so it runs in a
child process here) computes every column with the same expressions.  Fields,
the monitor DFT and the gradient (forward with curl record, reverse sweep) of
the two agree to rounding on a grid whose width spans two 64-column tiles with
a ragged, odd-width second tile, with the physical CPML axes and a probe."""

from __future__ import annotations

import os
import subprocess
import sys

import pytest
import torch

from conftest import ROOT, rel_l2

SHAPE = (22, 37, 101)

CHILD = r"""
import sys, torch
sys.path.insert(0, {root!r})
import diffnano_b200 as dn
shape = {shape!r}
g = torch.Generator().manual_seed(5)
eps = (1.5 + 2.0 * torch.rand(*shape, dtype=torch.float64, generator=g)).cuda()
w = torch.randn(*shape, dtype=torch.float64, generator=torch.Generator().manual_seed(6)).cuda()
mon = [{{"component": "Ey", "box": [[15, 16], [4, 33], [3, 99]], "wavelengths_nm": [1550.0]}}]
s = dn.FDTDSolver3D(grid_shape=shape, pml_layers=4, n_steps=70, device="cuda",
                    cpml_axes="physical", monitors=mon, backward="time_reversal")
src = {{"type": "gaussian_pulse", "plane": "xy", "z": 5, "component": "Ex"}}
e = eps.clone().requires_grad_(True)
r = s.forward(e, source=dict(src))
dft = r.metadata["monitors"][0]["dft"]
((r.field[1].double() * w).sum() + (dft.abs() ** 2).sum() * 1e-6).backward()
torch.save({{"field": r.field.detach().double().cpu(),
            "dft": torch.view_as_real(dft.detach()).cpu(), "grad": e.grad.cpu()}}, sys.argv[1])
"""


def _run(columns: str, path: str) -> dict:
    env = dict(os.environ, DN_FDTD3D_LANE_COLUMNS=columns)
    code = CHILD.format(root=ROOT, shape=SHAPE)
    r = subprocess.run([sys.executable, "-c", code, path], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return torch.load(path)


@pytest.mark.gpu
def test_two_column_step_matches_one_column_step(cuda, tmp_path):
    two = _run("2", str(tmp_path / "two.pt"))
    one = _run("1", str(tmp_path / "one.pt"))
    assert float(two["field"].abs().max()) > 0 and float(two["grad"].abs().max()) > 0
    assert rel_l2(two["field"], one["field"]) < 1e-7
    assert rel_l2(two["dft"], one["dft"]) < 1e-7
    assert rel_l2(two["grad"], one["grad"]) < 1e-7
