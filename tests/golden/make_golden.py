"""Generate the golden fixtures in this folder by running DiffNano itself.

Run once, in a container that has the reference checkout (read-only); its
location comes from ``DIFFNANO_REFERENCE`` (default ``/root/reference``)::

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py

It imports the reference's own ``FDTDSolver2D`` / ``FDTDSolver3D``
(``diffnano/solvers/fdtd2d.py``, ``fdtd3d.py``), runs them in FP64 on the CPU
on seeded inputs, and writes the inputs and outputs as ``.npz`` files.
Nothing at test time reads the reference; the tests read these files.
"""

from __future__ import annotations

import json
import math
import os
import sys
import time

import numpy as np
import torch

REF = os.environ.get("DIFFNANO_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REF)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from diffnano.solvers.fdtd2d import FDTDSolver2D  # noqa: E402  (reference)
from diffnano.solvers.fdtd3d import FDTDSolver3D  # noqa: E402  (reference)

from diffnano_b200.workloads import blob_design, gaussian_pulse_for_band  # noqa: E402

torch.set_num_threads(os.cpu_count() or 1)


def _seeded(shape, seed):
    g = torch.Generator().manual_seed(seed)
    return 1.5 + torch.rand(*shape, dtype=torch.float64, generator=g)


def _wave(solver, n, src):
    return np.array([float(solver._source_waveform(s, src)) for s in range(n)])


def tm2d_cfg0(meta):
    """256x256 TMz, 20-cell CPML, courant 0.5, 2000 steps, blob design."""
    mask = blob_design(128, seed=0, sigma_cells=3.0)
    eps = torch.full((256, 256), 2.085, dtype=torch.float64)
    eps[64:192, 64:192] = 2.085 + (12.1 - 2.085) * mask
    src = gaussian_pulse_for_band(1550.0, 200.0)
    src.update(row=30, probe=[226, 128])
    s = FDTDSolver2D(grid_shape=(256, 256), dl=20.0, wavelength_nm=1550.0, polarization="TM",
                     pml_layers=20, n_steps=2000, courant=0.5)
    t = time.perf_counter()
    with torch.no_grad():
        r = s.forward(eps, source=dict(src))
    wall = time.perf_counter() - t
    meta["tm2d_cfg0_wall_s"] = wall
    meta["tm2d_cfg0_gcells"] = 256 * 256 * 2000 / wall / 1e9
    np.savez_compressed(
        os.path.join(HERE, "tm2d_cfg0.npz"),
        design_mask=mask.numpy().astype(np.uint8),
        ez=r.field[0].numpy(),
        series=torch.stack(r.metadata["snapshots"]).numpy(),
        wave=_wave(s, 2000, src),
        source=json.dumps(src),
    )


def te2d(meta):
    """48x40 TE (non-square), 6-cell CPML, point source, probe.

    The reference's TE update grows exponentially (its curl signs give
    Hz_tt = +D^T D Hz), so two fixtures: 40 steps (values ~1e7, fine in FP32)
    and 300 steps (values ~1e87, FP64 only)."""
    eps = _seeded((48, 40), 11)
    src = {"type": "gaussian_pulse", "pos": [20, 15], "probe": [30, 25]}
    for name, T in (("te2d", 40), ("te2d_long", 300)):
        s = FDTDSolver2D(grid_shape=(48, 40), polarization="TE", pml_layers=6, n_steps=T)
        with torch.no_grad():
            r = s.forward(eps, source=dict(src))
        meta[name + "_max_abs"] = float(r.field.abs().max())
        np.savez_compressed(os.path.join(HERE, name + ".npz"), eps=eps.numpy(),
                            hz=r.field[0].numpy(),
                            series=torch.stack(r.metadata["snapshots"]).numpy(),
                            wave=_wave(s, T, src), source=json.dumps(src), n_steps=T)


def tm2d_cont(meta):
    """40x36 TMz continuous source on the default row, 4-cell CPML, 250 steps."""
    eps = _seeded((40, 36), 12)
    src = {"type": "continuous", "amplitude": 0.7}
    s = FDTDSolver2D(grid_shape=(40, 36), polarization="TM", pml_layers=4, n_steps=250,
                     dl=15.0, courant=0.6)
    with torch.no_grad():
        r = s.forward(eps, source=dict(src))
    np.savez_compressed(os.path.join(HERE, "tm2d_cont.npz"), eps=eps.numpy(),
                        ez=r.field[0].numpy(), wave=_wave(s, 250, src), source=json.dumps(src))


def fd3d_line(meta):
    """20^3, 4-cell CPML, 100 steps, default line source (reference axes)."""
    eps = _seeded((20, 20, 20), 13)
    eps[6:14, 6:14, 6:14] = 4.0
    src = {"type": "gaussian_pulse"}
    s = FDTDSolver3D(grid_shape=(20, 20, 20), pml_layers=4, n_steps=100)
    t = time.perf_counter()
    with torch.no_grad():
        r = s.forward(eps, source=dict(src))
    meta["fd3d_line_wall_s"] = time.perf_counter() - t
    np.savez_compressed(os.path.join(HERE, "fd3d_line.npz"), eps=eps.numpy(),
                        field=r.field.numpy(), wave=_wave(s, 100, src), source=json.dumps(src))


def fd3d_plane(meta):
    """16^3, 3-cell CPML, courant 0.35, xz-plane source, Ez probe series."""
    eps = _seeded((16, 16, 16), 14)
    src = {"type": "gaussian_pulse", "plane": "xz", "y": 5, "amplitude": 2.0}
    s = FDTDSolver3D(grid_shape=(16, 16, 16), pml_layers=3, n_steps=60, courant=0.35,
                     dl=25.0)
    with torch.no_grad():
        r = s.forward(eps, source=dict(src))
        ts = s.time_series(eps, probe=(8, 9, 7), source=dict(src))
    np.savez_compressed(os.path.join(HERE, "fd3d_plane.npz"), eps=eps.numpy(),
                        field=r.field.numpy(), series=ts.numpy(),
                        wave=_wave(s, 60, src), source=json.dumps(src))


def grad2d(meta):
    """dL/deps through the reference's autograd, 2-D TMz 24x20, 60 steps."""
    eps0 = _seeded((24, 20), 15)
    g = torch.Generator().manual_seed(16)
    G = torch.randn(1, 24, 20, dtype=torch.float64, generator=g)
    src = {"type": "gaussian_pulse", "row": 7}
    s = FDTDSolver2D(grid_shape=(24, 20), pml_layers=4, n_steps=60)
    eps = eps0.clone().requires_grad_(True)
    r = s.forward(eps, source=dict(src))
    (r.field * G).sum().backward()
    np.savez_compressed(os.path.join(HERE, "grad2d.npz"), eps=eps0.numpy(), G=G.numpy(),
                        ez=r.field.detach().numpy(), grad=eps.grad.numpy(),
                        source=json.dumps(src))


def grad3d(meta):
    """dL/deps, 3-D 10^3, 2-cell CPML, 30 steps: autograd and "time_reversal"."""
    eps0 = _seeded((10, 10, 10), 17)
    g = torch.Generator().manual_seed(18)
    G = torch.randn(3, 10, 10, 10, dtype=torch.float64, generator=g)
    src = {"type": "gaussian_pulse", "pos": [4, 5, 6]}
    out = {}
    for mode in ("auto", "time_reversal"):
        s = FDTDSolver3D(grid_shape=(10, 10, 10), pml_layers=2, n_steps=30, courant=0.35,
                         backward=mode)
        eps = eps0.clone().requires_grad_(True)
        r = s.forward(eps, source=dict(src))
        (r.field * G).sum().backward()
        out[mode] = eps.grad.clone()
        out["field"] = r.field.detach()
    meta["grad3d_tr_equals_ad"] = bool(torch.equal(out["auto"], out["time_reversal"]))
    np.savez_compressed(os.path.join(HERE, "grad3d.npz"), eps=eps0.numpy(), G=G.numpy(),
                        field=out["field"].numpy(), grad=out["auto"].numpy(),
                        grad_tr=out["time_reversal"].numpy(), source=json.dumps(src))


if __name__ == "__main__":
    meta = {"torch": torch.__version__, "threads": torch.get_num_threads()}
    for fn in (tm2d_cfg0, te2d, tm2d_cont, fd3d_line, fd3d_plane, grad2d, grad3d):
        t = time.perf_counter()
        fn(meta)
        print(f"{fn.__name__}: {time.perf_counter() - t:.2f} s", flush=True)
    meta["pi"] = math.pi
    with open(os.path.join(HERE, "golden_meta.json"), "w") as fh:
        json.dump(meta, fh, indent=1, sort_keys=True)
    print(json.dumps(meta, indent=1))
