"""GPU parity of the forward kernels against the reference's golden outputs
and the CPU FP64 oracle.

Tolerances (relative L2 of the whole field):
  * FP32 kernels vs the reference (FP64): 1e-5  (the target tolerance);
  * FP64 kernels vs the reference:        1e-12 (same algorithm, FMA and
    multiply-by-1/dl rounding only).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch
from conftest import DT2, DT3, OMEGA, cfg0_eps, load_golden, rel_l2

import diffnano_b200 as dn
from oracle import fdtd_ref as R

pytestmark = pytest.mark.gpu

TOL = {torch.float32: 1e-5, torch.float64: 1e-12}
DTYPES = [torch.float32, torch.float64]


@pytest.mark.parametrize("dtype", DTYPES)
def test_tm2d_cfg0_vs_reference(cuda, dtype):
    g = load_golden("tm2d_cfg0")
    s = dn.FDTDSolver2D(grid_shape=(256, 256), dl=20.0, wavelength_nm=1550.0, polarization="TM",
                        pml_layers=20, n_steps=2000, courant=0.5, device=cuda, dtype=dtype)
    r = s.forward(cfg0_eps(g["design_mask"]).to(cuda), source=dict(g["source"]))
    assert r.field.shape == (1, 256, 256) and r.field.dtype == dtype
    assert rel_l2(r.field[0], g["ez"]) < TOL[dtype]
    series = torch.stack(r.metadata["snapshots"])
    assert rel_l2(series, g["series"]) < TOL[dtype]


@pytest.mark.parametrize("name,dtype", [("te2d", torch.float32), ("te2d", torch.float64),
                                        ("te2d_long", torch.float64)])
def test_te2d_vs_reference(cuda, name, dtype):
    """The reference's TE scheme grows exponentially (to ~1e87 in the long
    fixture, beyond FP32's range), so FP32 is checked on the 40-step run."""
    g = load_golden(name)
    s = dn.FDTDSolver2D(grid_shape=(48, 40), polarization="TE", pml_layers=6,
                        n_steps=int(g["n_steps"]), device=cuda, dtype=dtype)
    r = s.forward(torch.tensor(g["eps"]), source=dict(g["source"]))
    assert rel_l2(r.field[0], g["hz"]) < TOL[dtype]
    assert rel_l2(torch.stack(r.metadata["snapshots"]), g["series"]) < TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
def test_tm2d_continuous_vs_reference(cuda, dtype):
    g = load_golden("tm2d_cont")
    s = dn.FDTDSolver2D(grid_shape=(40, 36), polarization="TM", pml_layers=4, n_steps=250,
                        dl=15.0, courant=0.6, device=cuda, dtype=dtype)
    r = s.forward(torch.tensor(g["eps"]).to(cuda), source=dict(g["source"]))
    assert rel_l2(r.field[0], g["ez"]) < TOL[dtype]


def test_2d_cpu_device_roundtrip(cuda):
    """device='cpu' (the reference's default): inputs/outputs on the host,
    kernels on the GPU."""
    g = load_golden("tm2d_cont")
    s = dn.FDTDSolver2D(grid_shape=(40, 36), pml_layers=4, n_steps=250, dl=15.0, courant=0.6)
    r = s.forward(torch.tensor(g["eps"]), source=dict(g["source"]))
    assert r.field.device.type == "cpu"
    assert rel_l2(r.field[0], g["ez"]) < 1e-5


@pytest.mark.parametrize("dtype", DTYPES)
def test_3d_line_vs_reference(cuda, dtype):
    g = load_golden("fd3d_line")
    s = dn.FDTDSolver3D(grid_shape=(20, 20, 20), pml_layers=4, n_steps=100, device=cuda,
                        dtype=dtype)
    r = s.forward(torch.tensor(g["eps"]).to(cuda), source=dict(g["source"]))
    assert r.field.shape == (3, 20, 20, 20)
    assert rel_l2(r.field, g["field"]) < TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
def test_3d_plane_and_time_series_vs_reference(cuda, dtype):
    g = load_golden("fd3d_plane")
    s = dn.FDTDSolver3D(grid_shape=(16, 16, 16), pml_layers=3, n_steps=60, courant=0.35,
                        dl=25.0, device=cuda, dtype=dtype)
    eps = torch.tensor(g["eps"]).to(cuda)
    r = s.forward(eps, source=dict(g["source"]))
    assert rel_l2(r.field, g["field"]) < TOL[dtype]
    ts = s.time_series(eps, probe=(8, 9, 7), source=dict(g["source"]))
    assert ts.shape == (60,)
    assert rel_l2(ts, g["series"]) < TOL[dtype]


def _seeded(shape, seed):
    gen = torch.Generator().manual_seed(seed)
    return 1.5 + 2.0 * torch.rand(*shape, dtype=torch.float64, generator=gen)


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("shape", [(40, 40, 40), (33, 33, 33)])
def test_3d_multi_tile_vs_oracle(cuda, dtype, shape):
    """Grids spanning several 16x32 tiles, ragged edges, several z ranges."""
    eps = _seeded(shape, 3)
    src = {"type": "gaussian_pulse", "pos": [shape[0] // 3, shape[1] // 2, shape[2] - 5]}
    T = 40
    o = R.run_3d(eps, dl=20.0, dt=DT3(0.4, 20.0), omega=OMEGA, pml_layers=5, n_steps=T,
                 source=src)
    s = dn.FDTDSolver3D(grid_shape=shape, pml_layers=5, n_steps=T, device=cuda, dtype=dtype)
    r = s.forward(eps.to(cuda), source=dict(src))
    ref = torch.stack([o["Ez"], o["Ex"], o["Ey"]])
    assert rel_l2(r.field, ref) < TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
def test_3d_physical_axes_non_cubic_vs_oracle(cuda, dtype):
    shape = (20, 24, 36)
    eps = _seeded(shape, 4)
    src = {"type": "gaussian_pulse", "plane": "xy", "z": 7, "component": "Ex"}
    T = 50
    o = R.run_3d(eps, dl=25.0, dt=DT3(0.4, 25.0), omega=OMEGA, pml_layers=4, n_steps=T,
                 source=src, axes="physical", component="Ex")
    s = dn.FDTDSolver3D(grid_shape=shape, dl=25.0, pml_layers=4, n_steps=T, device=cuda,
                        dtype=dtype, cpml_axes="physical")
    r = s.forward(eps.to(cuda), source=dict(src))
    ref = torch.stack([o["Ez"], o["Ex"], o["Ey"]])
    assert rel_l2(r.field, ref) < TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
def test_3d_monitors_vs_oracle(cuda, dtype):
    shape = (24, 24, 24)
    eps = _seeded(shape, 5)
    src = {"type": "gaussian_pulse", "plane": "xy", "z": 6, "component": "Ex",
           "spread": 900.0, "t0": 2700.0}
    wl = [1500.0, 1550.0, 1600.0]
    mons = [{"component": "Ey", "plane": "xy", "z": 17, "extent": [[4, 20], [2, 22]],
             "wavelengths_nm": wl},
            {"component": "Hz", "pos": [12, 12, 12], "wavelengths_nm": [1550.0]}]
    T = 120
    omon = [dict(component="Ey", box=((17, 18), (4, 20), (2, 22)), wavelengths_nm=wl),
            dict(component="Hz", box=((12, 13), (12, 13), (12, 13)), wavelengths_nm=[1550.0])]
    o = R.run_3d(eps, dl=20.0, dt=DT3(0.4, 20.0), omega=OMEGA, pml_layers=4, n_steps=T,
                 source=src, monitors=omon, component="Ex")
    s = dn.FDTDSolver3D(grid_shape=shape, pml_layers=4, n_steps=T, device=cuda, dtype=dtype)
    r = s.forward(eps.to(cuda), source=dict(src), monitors=mons)
    got = r.metadata["monitors"]
    for m in range(2):
        ref = torch.view_as_complex(o["monitors"][m].contiguous())
        assert got[m]["dft"].shape == ref.shape
        assert rel_l2(torch.view_as_real(got[m]["dft"]), torch.view_as_real(ref)) < TOL[dtype] * 10


@pytest.mark.parametrize("pol", ["TM", "TE"])
def test_2d_monitors_vs_oracle(cuda, pol):
    g = load_golden("tm2d_cont")
    eps = torch.tensor(g["eps"])
    comp = "Ez" if pol == "TM" else "Hz"
    wl = [1450.0, 1550.0, 1650.0]
    src = {"type": "gaussian_pulse", "row": 6}
    T = 250 if pol == "TM" else 40  # the reference's TE scheme grows exponentially
    o = R.run_2d(eps, dl=15.0, dt=DT2(0.6, 15.0), omega=OMEGA, pml_layers=4, polarization=pol,
                 n_steps=T, source=src,
                 monitors=[dict(component=comp, box=((30, 31), (0, 36)), wavelengths_nm=wl)])
    s = dn.FDTDSolver2D(grid_shape=(40, 36), polarization=pol, pml_layers=4, n_steps=T,
                        dl=15.0, courant=0.6, device=cuda, dtype=torch.float64)
    r = s.forward(eps, source=dict(src), monitors=[{"component": comp, "row": 30,
                                                    "wavelengths_nm": wl}])
    ref = torch.view_as_complex(o["monitors"][0].contiguous())
    got = r.metadata["monitors"][0]["dft"]
    assert rel_l2(torch.view_as_real(got), torch.view_as_real(ref)) < 1e-11


@pytest.mark.parametrize("pol,dtype", [("TM", torch.float32), ("TE", torch.float32),
                                       ("TM", torch.float64), ("TE", torch.float64)])
def test_2d_unaligned_rows_match_padded_rows(cuda, pol, dtype):
    """The 2-D step through the C ABI with tight rows (pitch = W = 45: rows
    not on 16-byte boundaries, one value per lane) against the engine's
    padded rows (16-byte row access, with a partly filled last lane)."""
    import ctypes

    from diffnano_b200 import _lib
    from diffnano_b200.solvers import _setup
    from diffnano_b200.solvers._engine import Engine

    H, W, T = 70, 45, 40
    dl, courant = 20.0, 0.5
    dt = courant * dl / 2 ** 0.5
    src = {"type": "gaussian_pulse", "row": 9, "spread": 500.0, "t0": 800.0}
    p = _lib.DN_TM if pol == "TM" else _lib.DN_TE
    comp = _lib.DN_EZ if pol == "TM" else _lib.DN_HZ
    eng = Engine(is3d=False, shape=(H, W), dl=dl, dt=dt, pml_layers=6, dtype=dtype, device=cuda,
                 n_steps=T, wave=_setup.waveform_table(T, dt, OMEGA, src),
                 src_box=_setup.source_box_2d((H, W), src), src_comp=comp, pol=p)
    g = torch.Generator().manual_seed(11)
    eng.set_eps(1.5 + 2.0 * torch.rand(H, W, dtype=torch.float64, generator=g))
    assert eng.Wp != W and (eng.Wp * eng.A.element_size()) % 16 == 0
    eng.run(0, T)

    grid = type(eng.grid).from_buffer_copy(eng.grid)
    grid.pitch_y, grid.pitch_z = W, H * W
    fa = torch.zeros((6, H, W), dtype=dtype, device=cuda)
    fb = torch.zeros_like(fa)
    ce = eng.ce[0, :, :W].contiguous()
    assert (W * fa.element_size()) % 16 != 0
    out = ctypes.c_int32(0)
    with torch.cuda.device(cuda):
        stream = torch.cuda.current_stream(cuda).cuda_stream
        rc = _lib.lib().dn_fdtd2d_run(
            ctypes.byref(grid), _lib.PTR6(*[fa[c].data_ptr() for c in range(6)]),
            _lib.PTR6(*[fb[c].data_ptr() for c in range(6)]), ce.data_ptr(),
            ctypes.byref(eng.cpml), ctypes.byref(eng.src), None, 0,
            ctypes.byref(_lib.DnProbe(component=_lib.DN_NONE)), None, 0, T,
            eng.status.data_ptr(), ctypes.c_void_p(stream), ctypes.byref(out))
    assert rc == _lib.DN_OK
    eng.check_status()
    res = fb if out.value else fa
    tol = 1e-6 if dtype == torch.float32 else 1e-13
    comps = (_lib.DN_EZ, _lib.DN_HX, _lib.DN_HY) if pol == "TM" else \
        (_lib.DN_HZ, _lib.DN_EX, _lib.DN_EY)
    for c in comps:
        ref = eng.field(c)[0]
        assert float(ref.abs().max()) > 0
        assert rel_l2(res[c], ref) < tol


@pytest.mark.parametrize("pol", ["TM", "TE"])
def test_2d_large_grid_vs_oracle(cuda, pol):
    """1024^2: the per-step kernel marches 4 rows per warp here (the smaller
    grids of the other tests march 2).  FP32 against the FP64 oracle."""
    n, T = 1024, 30
    g = torch.Generator().manual_seed(5)
    eps = 1.5 + 2.0 * torch.rand(n, n, dtype=torch.float64, generator=g)
    src = {"type": "gaussian_pulse", "row": 30, "t0": 40.0, "spread": 20.0}
    o = R.run_2d(eps, dl=20.0, dt=DT2(0.5, 20.0), omega=OMEGA, pml_layers=20, polarization=pol,
                 n_steps=T, source=dict(src))
    s = dn.FDTDSolver2D(grid_shape=(n, n), polarization=pol, pml_layers=20, n_steps=T,
                        dl=20.0, courant=0.5, device=cuda, dtype=torch.float32)
    # a probe keeps the solve on the per-step kernel (no cluster-resident path)
    r = s.forward(eps.to(cuda), source=dict(src, probe=[n // 2, n // 2]))
    comp = "Ez" if pol == "TM" else "Hz"
    assert float(o[comp].abs().max()) > 0
    assert rel_l2(r.field[0], o[comp]) < 1e-5


def test_2d_large_grid_gradient_vs_oracle(cuda):
    """1024^2 TM gradient (forward with curl record, 4-row warp marches in both
    directions) against the oracle's autograd, FP64."""
    n, T = 1024, 20
    g = torch.Generator().manual_seed(6)
    eps0 = 1.5 + 2.0 * torch.rand(n, n, dtype=torch.float64, generator=g)
    src = {"type": "gaussian_pulse", "row": 30, "t0": 40.0, "spread": 20.0}
    e = eps0.clone().requires_grad_(True)
    o = R.run_2d(e, dl=20.0, dt=DT2(0.5, 20.0), omega=OMEGA, pml_layers=20, n_steps=T,
                 source=dict(src))
    (o["Ez"] * o["Ez"]).sum().backward()
    s = dn.FDTDSolver2D(grid_shape=(n, n), pml_layers=20, n_steps=T, dl=20.0, courant=0.5,
                        device=cuda, dtype=torch.float64)
    eps = eps0.clone().to(cuda).requires_grad_(True)
    r = s.forward(eps, source=dict(src))
    (r.field[0] * r.field[0]).sum().backward()
    assert float(e.grad.norm()) > 0
    assert rel_l2(eps.grad, e.grad) < 1e-9


def test_2d_engine_reuse_keeps_results_independent(cuda):
    """Gradient-free per-step solves reuse one engine per set-up: results of
    earlier calls (field, probe snapshots, DFTs) stay as they were, and the
    same input gives the same output again."""
    n = 96
    g = torch.Generator().manual_seed(8)
    e1 = (1.5 + 2.0 * torch.rand(n, n, dtype=torch.float64, generator=g)).to(cuda)
    e2 = (1.5 + 2.0 * torch.rand(n, n, dtype=torch.float64, generator=g)).to(cuda)
    src = {"type": "gaussian_pulse", "row": 10, "probe": [60, 40]}
    mons = [{"component": "Ez", "row": 70, "wavelengths_nm": [1500.0, 1600.0]}]
    s = dn.FDTDSolver2D(grid_shape=(n, n), pml_layers=6, n_steps=120, device=cuda,
                        monitors=mons)
    r1 = s.forward(e1, source=dict(src))
    f1 = r1.field.clone()
    p1 = torch.stack(r1.metadata["snapshots"]).clone()
    d1 = r1.metadata["monitors"][0]["dft"].clone()
    r2 = s.forward(e2, source=dict(src))
    r3 = s.forward(e1, source=dict(src))
    assert len(s.__dict__.get("_engine_cache", {})) == 1
    assert not torch.equal(r2.field, f1)
    assert torch.equal(r1.field, f1) and torch.equal(torch.stack(r1.metadata["snapshots"]), p1)
    assert torch.equal(r1.metadata["monitors"][0]["dft"], d1)
    assert torch.equal(r3.field, f1) and torch.equal(torch.stack(r3.metadata["snapshots"]), p1)
    assert torch.equal(r3.metadata["monitors"][0]["dft"], d1)


def test_deterministic(cuda):
    shape = (32, 32, 32)
    eps = _seeded(shape, 6).to(cuda)
    s = dn.FDTDSolver3D(grid_shape=shape, pml_layers=4, n_steps=30, device=cuda)
    a = s.forward(eps).field
    b = s.forward(eps).field
    assert torch.equal(a, b)


def test_time_step_hook_matches_oracle(cuda):
    """The private one-step hook the reference's bandwidth harness calls."""
    shape = (12, 12, 12)
    gen = torch.Generator().manual_seed(7)
    f = [torch.randn(*shape, dtype=torch.float64, generator=gen) for _ in range(6)]
    eps = _seeded(shape, 8)
    s = dn.FDTDSolver3D(grid_shape=shape, pml_layers=3, device=cuda, dtype=torch.float64)
    got = s._time_step(*(t.to(cuda) for t in f), eps.to(cuda), torch.ones_like(eps).to(cuda))
    prof = (*R.cpml_profile(12, 3, 20.0, s.dt),) * 3
    ref = R.step_3d(*f, eps, prof, s.dt, 20.0)
    for a, b in zip(got, ref):
        assert rel_l2(a, b) < 1e-13
