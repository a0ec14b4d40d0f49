"""Parity at the 3-D benchmark configuration itself.

The benchmark's 3-D line is quoted on 256^3 cells, dl 25 nm, a 12-cell CPML,
Courant 0.4 and a 4000-step solve, with an Ex-polarised Gaussian plane
source at z = 40 and an Ey DFT monitor on a 64 x 64 plane at z = 200.  These
tests check the kernels on exactly that grid (``bench.workload()``), where
the work plan differs from every small grid: 128 tiles x 2 z ranges of 128
planes, the 4-stage ring wrapping around 32 times per range, and FP32
rounding accumulated over 4000 steps with a DFT added at every step.

* FP32 kernels against the FP64 build of the same kernels over the whole
  4000-step solve: fields and monitor DFT.
* Both builds against the CPU FP64 oracle at full width: 20 steps from a
  seeded random state in every cell of all six fields (so every plane, tile
  edge, z-range seam and CPML face carries a non-zero value), source and
  monitor on, starting at step 1000 (near the pulse peak).
* dL/deps of L = sum |DFT Ey|^2 at 16 seeded voxels of the design block
  against central finite differences (h = 1e-3) of the FP64 kernels -- the
  check the 3-D configuration itself specifies.
* The FP32 gradient against the FP64 gradient over the whole grid.

Tolerances (relative L2): fields 1e-5 (FP32) and 1e-12 (FP64) against the
oracle; FP32 vs FP64 fields 1e-5 and DFT 1e-5; gradients 1e-4 against finite
differences and FP32 vs FP64.  The measured values are printed (run with
``-s`` to see them).
"""

from __future__ import annotations

import math
import os

import pytest
import torch
from conftest import rel_l2

import bench
import diffnano_b200 as dn
from oracle import fdtd_ref as R

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

_CACHE: dict = {}
DESIGN_Z = (96, 136)   # slab_eps_3d: substrate 3*256//8 = 96 cells, 40-cell block
DESIGN_YX = (64, 192)  # 128 x 128 block centred in y and x


@pytest.fixture(scope="module")
def cfg1():
    eps, src, mons = bench.workload()
    assert tuple(eps.shape) == bench.SHAPE == (256, 256, 256)
    return eps, src, mons


def _solver(cuda, dtype, **kw):
    return dn.FDTDSolver3D(grid_shape=bench.SHAPE, dl=bench.DL, wavelength_nm=1550.0,
                           pml_layers=bench.PML, n_steps=bench.T_SOLVE, courant=bench.COURANT,
                           device=cuda, dtype=dtype, **kw)


def _fom(r):
    return (r.metadata["monitors"][0]["dft"].abs() ** 2).sum()


def _forward(cuda, cfg, dtype):
    key = ("fwd", dtype)
    if key not in _CACHE:
        eps, src, mons = cfg
        with torch.no_grad():
            r = _solver(cuda, dtype).forward(eps.to(cuda), source=dict(src), monitors=mons)
        _CACHE[key] = (r.field.double().cpu(), r.metadata["monitors"][0]["dft"].cpu())
        del r
        torch.cuda.empty_cache()
    return _CACHE[key]


def _gradient(cuda, cfg, dtype):
    key = ("grad", dtype)
    if key not in _CACHE:
        eps, src, mons = cfg
        e = eps.clone().to(cuda).requires_grad_(True)
        L = _fom(_solver(cuda, dtype).forward(e, source=dict(src), monitors=mons))
        L.backward()
        _CACHE[key] = (float(L.detach()), e.grad.double().cpu())
        del e, L
        torch.cuda.empty_cache()
    return _CACHE[key]


def test_fp32_vs_fp64_kernels_full_solve(cuda, cfg1):
    f64, d64 = _forward(cuda, cfg1, torch.float64)
    f32, d32 = _forward(cuda, cfg1, torch.float32)
    assert float(f64.abs().max()) > 0 and float(d64.abs().max()) > 0
    assert torch.isfinite(f32).all() and torch.isfinite(d32).all()
    e_field, e_dft = rel_l2(f32, f64), rel_l2(d32, d64)
    print(f"\n256^3 x 4000 FP32 vs FP64 kernels: field rel-L2 {e_field:.3e}, "
          f"Ey DFT rel-L2 {e_dft:.3e}")
    assert e_field < 1e-5
    assert e_dft < 1e-5


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_full_width_vs_oracle(cuda, cfg1, dtype):
    eps, src, mons = cfg1
    D, H, W = bench.SHAPE
    t0, n = 1000, 20
    names = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
    eng = _solver(cuda, dtype)._make_engine(t0 + n, src, mons)
    box = eng.monitors[0].box
    assert box == ((200, 201), (96, 160), (96, 160))
    if "oracle" not in _CACHE:
        gen = torch.Generator().manual_seed(11)
        init = {k: torch.randn(D, H, W, dtype=torch.float64, generator=gen) for k in names}
        torch.set_num_threads(os.cpu_count() or 1)
        o = R.run_3d(eps, dl=bench.DL, dt=bench.COURANT * bench.DL / math.sqrt(3.0),
                     omega=2 * math.pi / 1550.0, pml_layers=bench.PML, n_steps=n, source=src,
                     monitors=[{"component": "Ey", "box": box, "wavelengths_nm": [1550.0]}],
                     component="Ex", init=init, t0=t0)
        _CACHE["oracle"] = (init, o)
    init, o = _CACHE["oracle"]
    eng.set_eps(eps.to(cuda))
    for k in names:
        eng.field(dn._lib.COMPONENTS[k]).copy_(init[k].to(cuda))
    eng.run(t0, n)
    eng.check_status()
    tol = 1e-5 if dtype == torch.float32 else 1e-12
    errs = {k: rel_l2(eng.field(dn._lib.COMPONENTS[k]), o[k]) for k in names}
    dft = eng.monitor_dft(0)
    e_dft = rel_l2(torch.view_as_real(dft.cpu()).reshape(o["monitors"][0].shape),
                   o["monitors"][0])
    print(f"\n256^3 from a random state, steps {t0}..{t0 + n - 1}, {dtype}: "
          + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()) + f", Ey DFT {e_dft:.2e}")
    for k, v in errs.items():
        assert v < tol, (k, v)
    assert e_dft < tol
    del eng
    torch.cuda.empty_cache()


def test_gradient_vs_central_differences_16_voxels(cuda, cfg1):
    """The 3-D configuration's own gradient check, on the FP64 kernels."""
    eps, src, mons = cfg1
    L0, g64 = _gradient(cuda, cfg1, torch.float64)
    s = _solver(cuda, torch.float64)
    gen = torch.Generator().manual_seed(16)
    vox = torch.stack([torch.randint(*DESIGN_Z, (16,), generator=gen),
                       torch.randint(*DESIGN_YX, (16,), generator=gen),
                       torch.randint(*DESIGN_YX, (16,), generator=gen)], 1)
    h = 1e-3
    fd, ad = [], []
    with torch.no_grad():
        for z, y, x in vox.tolist():
            vals = []
            for sign in (1.0, -1.0):
                e = eps.clone()
                e[z, y, x] += sign * h
                vals.append(float(_fom(s.forward(e.to(cuda), source=dict(src), monitors=mons))))
            fd.append((vals[0] - vals[1]) / (2 * h))
            ad.append(float(g64[z, y, x]))
    fd_t, ad_t = torch.tensor(fd, dtype=torch.float64), torch.tensor(ad, dtype=torch.float64)
    err = rel_l2(ad_t, fd_t)
    print(f"\n256^3 x 4000 FP64 FOM {L0:.6e}; adjoint vs central FD at 16 voxels: rel-L2 "
          f"{err:.3e}; max |g| {float(fd_t.abs().max()):.3e}")
    assert float(fd_t.abs().max()) > 0
    assert err < 1e-4


def test_gradient_fp32_vs_fp64_full_grid(cuda, cfg1):
    L64, g64 = _gradient(cuda, cfg1, torch.float64)
    L32, g32 = _gradient(cuda, cfg1, torch.float32)
    assert torch.isfinite(g32).all()
    err = rel_l2(g32, g64)
    z0, z1 = DESIGN_Z
    y0, y1 = DESIGN_YX
    err_blk = rel_l2(g32[z0:z1, y0:y1, y0:y1], g64[z0:z1, y0:y1, y0:y1])
    print(f"\n256^3 x 4000 FOM FP32 {L32:.9e} vs FP64 {L64:.9e} (rel {abs(L32 / L64 - 1):.2e}); "
          f"dL/deps FP32 vs FP64 rel-L2 {err:.3e} (design block {err_blk:.3e})")
    assert abs(L32 / L64 - 1) < 1e-5
    assert err < 1e-4
    assert err_blk < 1e-4


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_non_cubic_full_width_vs_oracle(cuda, dtype):
    """A 128 x 256 x 256 grid with the physical CPML axes (128 tiles x 2 z
    ranges of 64 planes), 12 steps from a random state in every cell against
    the oracle, source and monitor on."""
    shape = (128, 256, 256)
    D, H, W = shape
    gen = torch.Generator().manual_seed(21)
    eps = 1.5 + 2.0 * torch.rand(*shape, dtype=torch.float64, generator=gen)
    src = {"type": "gaussian_pulse", "plane": "xy", "z": 20, "component": "Ex"}
    mons = [{"component": "Ez", "plane": "xy", "z": 100, "extent": [[40, 200], [30, 220]],
             "wavelengths_nm": [1500.0, 1600.0]}]
    names = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
    init = {k: torch.randn(*shape, dtype=torch.float64, generator=gen) for k in names}
    t0, n = 600, 12
    s = dn.FDTDSolver3D(grid_shape=shape, dl=25.0, pml_layers=12, n_steps=t0 + n, device=cuda,
                        dtype=dtype, cpml_axes="physical")
    eng = s._make_engine(t0 + n, src, mons)
    torch.set_num_threads(os.cpu_count() or 1)
    o = R.run_3d(eps, dl=25.0, dt=s.dt, omega=s.omega, pml_layers=12, n_steps=n, source=src,
                 monitors=[{"component": "Ez", "box": eng.monitors[0].box,
                            "wavelengths_nm": [1500.0, 1600.0]}],
                 axes="physical", component="Ex", init=init, t0=t0)
    eng.set_eps(eps.to(cuda))
    for k in names:
        eng.field(dn._lib.COMPONENTS[k]).copy_(init[k].to(cuda))
    eng.run(t0, n)
    eng.check_status()
    tol = 1e-5 if dtype == torch.float32 else 1e-12
    for k in names:
        assert rel_l2(eng.field(dn._lib.COMPONENTS[k]), o[k]) < tol, k
    dft = torch.view_as_real(eng.monitor_dft(0).cpu()).reshape(o["monitors"][0].shape)
    assert rel_l2(dft, o["monitors"][0]) < tol
