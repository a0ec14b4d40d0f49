"""The CPU FP64 oracle reproduces the reference's own outputs.

The fixtures in tests/golden/ were produced by running DiffNano's
FDTDSolver2D / FDTDSolver3D (make_golden.py).  The oracle must match them
bit for bit (fields, probe series, waveform tables) and gradients to 1e-13
(autograd's accumulation order may differ in the last bit).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch
from conftest import DT2, DT3, OMEGA, cfg0_eps, load_golden, rel_l2

from oracle import fdtd_ref as R


def test_waveform_cfg0_bit_exact():
    g = load_golden("tm2d_cfg0")
    w = R.waveform_table(2000, DT2(0.5, 20.0), OMEGA, g["source"]).numpy()
    assert np.array_equal(w, g["wave"])


def test_tm2d_cfg0_bit_exact():
    g = load_golden("tm2d_cfg0")
    src = g["source"]
    o = R.run_2d(cfg0_eps(g["design_mask"]), dl=20.0, dt=DT2(0.5, 20.0), omega=OMEGA,
                 pml_layers=20, n_steps=2000, source=src, probe=src["probe"])
    assert np.array_equal(o["Ez"].numpy(), g["ez"])
    assert np.array_equal(o["series"].numpy(), g["series"])


@pytest.mark.parametrize("name", ["te2d", "te2d_long"])
def test_te2d_bit_exact(name):
    """TE, including the 300-step run where the reference's TE scheme has
    grown to ~1e87 (its curl signs make TE exponentially unstable)."""
    g = load_golden(name)
    src = g["source"]
    o = R.run_2d(torch.tensor(g["eps"]), dl=20.0, dt=DT2(0.5, 20.0), omega=OMEGA, pml_layers=6,
                 polarization="TE", n_steps=int(g["n_steps"]), source=src, probe=src["probe"])
    assert np.array_equal(o["Hz"].numpy(), g["hz"])
    assert np.array_equal(o["series"].numpy(), g["series"])


def test_tm2d_continuous_bit_exact():
    g = load_golden("tm2d_cont")
    o = R.run_2d(torch.tensor(g["eps"]), dl=15.0, dt=DT2(0.6, 15.0), omega=OMEGA, pml_layers=4,
                 n_steps=250, source=g["source"])
    assert np.array_equal(o["Ez"].numpy(), g["ez"])
    assert np.array_equal(R.waveform_table(250, DT2(0.6, 15.0), OMEGA, g["source"]).numpy(),
                          g["wave"])


def test_3d_line_bit_exact():
    g = load_golden("fd3d_line")
    o = R.run_3d(torch.tensor(g["eps"]), dl=20.0, dt=DT3(0.4, 20.0), omega=OMEGA, pml_layers=4,
                 n_steps=100, source=g["source"])
    f = torch.stack([o["Ez"], o["Ex"], o["Ey"]]).numpy()
    assert np.array_equal(f, g["field"])


def test_3d_plane_and_series_bit_exact():
    g = load_golden("fd3d_plane")
    o = R.run_3d(torch.tensor(g["eps"]), dl=25.0, dt=DT3(0.35, 25.0), omega=OMEGA,
                 pml_layers=3, n_steps=60, source=g["source"], probe=(8, 9, 7))
    f = torch.stack([o["Ez"], o["Ex"], o["Ey"]]).numpy()
    assert np.array_equal(f, g["field"])
    assert np.array_equal(o["series"].numpy(), g["series"])


def test_grad2d_matches_reference_autograd():
    g = load_golden("grad2d")
    eps = torch.tensor(g["eps"]).requires_grad_(True)
    o = R.run_2d(eps, dl=20.0, dt=DT2(0.5, 20.0), omega=OMEGA, pml_layers=4, n_steps=60,
                 source=g["source"])
    (o["Ez"].unsqueeze(0) * torch.tensor(g["G"])).sum().backward()
    assert rel_l2(eps.grad, g["grad"]) < 1e-13


def test_grad3d_matches_reference_autograd_and_time_reversal():
    g = load_golden("grad3d")
    assert np.array_equal(g["grad"], g["grad_tr"])  # the reference's "TR" is autograd
    eps = torch.tensor(g["eps"]).requires_grad_(True)
    o = R.run_3d(eps, dl=20.0, dt=DT3(0.35, 20.0), omega=OMEGA, pml_layers=2, n_steps=30,
                 source=g["source"])
    (torch.stack([o["Ez"], o["Ex"], o["Ey"]]) * torch.tensor(g["G"])).sum().backward()
    assert rel_l2(eps.grad, g["grad"]) < 1e-13


def test_point_monitor_equals_dft_of_reference_series():
    """A point DFT monitor is the DFT of the reference's time series."""
    g = load_golden("te2d")
    src = g["source"]
    wl = [1500.0, 1600.0]
    py, px = src["probe"]
    T = int(g["n_steps"])
    o = R.run_2d(torch.tensor(g["eps"]), dl=20.0, dt=DT2(0.5, 20.0), omega=OMEGA, pml_layers=6,
                 polarization="TE", n_steps=T, source=src,
                 monitors=[dict(component="Hz", box=((py, py + 1), (px, px + 1)),
                                wavelengths_nm=wl)])
    dt = DT2(0.5, 20.0)
    n = np.arange(T)
    for li, lam in enumerate(wl):
        w = 2 * np.pi / lam
        ref = np.sum(g["series"] * np.exp(-1j * w * n * dt)) * dt
        got = o["monitors"][0][li, 0, 0]
        assert abs(complex(got[0], got[1]) - ref) <= 1e-12 * abs(ref)


def test_3d_restart_from_state_equals_one_run():
    """run_3d(init=state at step a, t0=a) continues an uninterrupted run bit
    for bit: fields exactly, monitor DFT as the remaining steps' share."""
    g = load_golden("fd3d_plane")
    kw = dict(dl=25.0, dt=DT3(0.35, 25.0), omega=OMEGA, pml_layers=3, source=g["source"])
    mon = [{"component": "Ey", "box": ((10, 11), (2, 14), (3, 13)), "wavelengths_nm": [1550.0]}]
    eps = torch.tensor(g["eps"])
    full = R.run_3d(eps, n_steps=60, monitors=mon, **kw)
    head = R.run_3d(eps, n_steps=25, monitors=mon, **kw)
    tail = R.run_3d(eps, n_steps=35, monitors=mon, init=head, t0=25, **kw)
    for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        assert torch.equal(tail[k], full[k]), k
    assert rel_l2(head["monitors"][0] + tail["monitors"][0], full["monitors"][0]) < 1e-15
