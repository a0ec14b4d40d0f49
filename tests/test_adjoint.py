"""GPU gradients (hand-written discrete adjoint) against the reference's
autograd (golden fixtures), the oracle's autograd and central finite
differences of the FP64 kernels.

Tolerances (relative L2 of dL/deps): FP64 kernels 1e-9 (same algorithm,
rounding only); FP32 kernels 1e-4 (the target); finite differences 1e-4.
"""

from __future__ import annotations

import pytest
import torch
from conftest import DT2, DT3, OMEGA, load_golden, rel_l2

import diffnano_b200 as dn
from oracle import fdtd_ref as R

pytestmark = pytest.mark.gpu

TOL = {torch.float32: 1e-4, torch.float64: 1e-9}
DTYPES = [torch.float32, torch.float64]


def _seeded(shape, seed, lo=1.5, span=2.0):
    g = torch.Generator().manual_seed(seed)
    return lo + span * torch.rand(*shape, dtype=torch.float64, generator=g)


@pytest.mark.parametrize("dtype", DTYPES)
def test_grad2d_tm_vs_reference_autograd(cuda, dtype):
    g = load_golden("grad2d")
    s = dn.FDTDSolver2D(grid_shape=(24, 20), pml_layers=4, n_steps=60, device=cuda, dtype=dtype)
    eps = torch.tensor(g["eps"]).to(cuda).requires_grad_(True)
    r = s.forward(eps, source=dict(g["source"]))
    (r.field.double() * torch.tensor(g["G"]).to(cuda)).sum().backward()
    assert eps.grad.dtype == torch.float64
    assert rel_l2(eps.grad, g["grad"]) < TOL[dtype]


@pytest.mark.parametrize("mode", ["auto", "time_reversal", "checkpoint"])
@pytest.mark.parametrize("dtype", DTYPES)
def test_grad3d_vs_reference_autograd(cuda, dtype, mode):
    g = load_golden("grad3d")
    kw = dict(use_checkpoint=True, checkpoint_segments=4) if mode == "checkpoint" else \
        dict(backward=mode)
    s = dn.FDTDSolver3D(grid_shape=(10, 10, 10), pml_layers=2, n_steps=30, courant=0.35,
                        device=cuda, dtype=dtype, **kw)
    eps = torch.tensor(g["eps"]).to(cuda).requires_grad_(True)
    r = s.forward(eps, source=dict(g["source"]))
    if mode == "time_reversal":
        assert "TimeReversalFDTD" in type(r.field.grad_fn).__name__ or \
            "TimeReversalFDTD" in str(r.field.grad_fn.next_functions)
    (r.field.double() * torch.tensor(g["G"]).to(cuda)).sum().backward()
    assert rel_l2(eps.grad, g["grad"]) < TOL[dtype]


def test_grad_on_cpu_tensor_roundtrip(cuda):
    """device='cpu' solver: eps and its gradient stay on the host."""
    g = load_golden("grad3d")
    s = dn.FDTDSolver3D(grid_shape=(10, 10, 10), pml_layers=2, n_steps=30, courant=0.35,
                        dtype=torch.float64, backward="time_reversal")
    eps = torch.tensor(g["eps"]).requires_grad_(True)
    r = s.forward(eps, source=dict(g["source"]))
    (r.field * torch.tensor(g["G"])).sum().backward()
    assert eps.grad.device.type == "cpu"
    assert rel_l2(eps.grad, g["grad"]) < 1e-9


@pytest.mark.parametrize("dtype", DTYPES)
def test_grad2d_te_vs_oracle(cuda, dtype):
    shape, T = (26, 34), 24
    eps0 = _seeded(shape, 21)
    src = {"type": "gaussian_pulse", "pos": [12, 15]}
    G = torch.randn(*shape, dtype=torch.float64, generator=torch.Generator().manual_seed(22))
    e = eps0.clone().requires_grad_(True)
    o = R.run_2d(e, dl=20.0, dt=DT2(0.5, 20.0), omega=OMEGA, pml_layers=4, polarization="TE",
                 n_steps=T, source=src)
    (o["Hz"] * G).sum().backward()
    s = dn.FDTDSolver2D(grid_shape=shape, polarization="TE", pml_layers=4, n_steps=T,
                        device=cuda, dtype=dtype)
    eps = eps0.clone().to(cuda).requires_grad_(True)
    r = s.forward(eps, source=dict(src))
    (r.field[0].double() * G.to(cuda)).sum().backward()
    assert rel_l2(eps.grad, e.grad) < TOL[dtype] * 10  # TE grows exponentially


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("shape,axes", [((18, 18, 18), "reference"), ((20, 24, 36), "physical"),
                                        ((33, 40, 35), "physical")])
def test_grad3d_vs_oracle(cuda, dtype, shape, axes):
    """Multi-tile / ragged grids, both CPML mappings, Ex plane source,
    several checkpoint segments (T not a multiple of the interval)."""
    T = 29
    eps0 = _seeded(shape, 23)
    src = {"type": "gaussian_pulse", "plane": "xy", "z": 5, "component": "Ex",
           "spread": 300.0, "t0": 900.0}
    G = torch.randn(3, *shape, dtype=torch.float64, generator=torch.Generator().manual_seed(24))
    e = eps0.clone().requires_grad_(True)
    o = R.run_3d(e, dl=20.0, dt=DT3(0.4, 20.0), omega=OMEGA, pml_layers=4, n_steps=T,
                 source=src, axes=axes, component="Ex")
    (torch.stack([o["Ez"], o["Ex"], o["Ey"]]) * G).sum().backward()
    s = dn.FDTDSolver3D(grid_shape=shape, pml_layers=4, n_steps=T, device=cuda, dtype=dtype,
                        cpml_axes=axes)
    eps = eps0.clone().to(cuda).requires_grad_(True)
    r = s.forward(eps, source=dict(src))
    (r.field.double() * G.to(cuda)).sum().backward()
    assert rel_l2(eps.grad, e.grad) < TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
def test_monitor_fom_gradient_vs_oracle(cuda, dtype):
    """Loss = sum |DFT Ey|^2 over a plane monitor (the 3-D workload's FOM)."""
    shape, T = (22, 22, 22), 60
    eps0 = _seeded(shape, 25)
    src = {"type": "gaussian_pulse", "plane": "xy", "z": 5, "component": "Ex",
           "spread": 400.0, "t0": 1200.0}
    wl = [1500.0, 1600.0]
    e = eps0.clone().requires_grad_(True)
    o = R.run_3d(e, dl=20.0, dt=DT3(0.4, 20.0), omega=OMEGA, pml_layers=3, n_steps=T,
                 source=src, component="Ex",
                 monitors=[dict(component="Ey", box=((16, 17), (4, 18), (3, 19)),
                                wavelengths_nm=wl)])
    R.fom_abs2(o["monitors"][0]).backward()
    s = dn.FDTDSolver3D(grid_shape=shape, pml_layers=3, n_steps=T, device=cuda, dtype=dtype)
    eps = eps0.clone().to(cuda).requires_grad_(True)
    r = s.forward(eps, source=dict(src),
                  monitors=[{"component": "Ey", "plane": "xy", "z": 16,
                             "extent": [[4, 18], [3, 19]], "wavelengths_nm": wl}])
    F = r.metadata["monitors"][0]["dft"]
    (F.abs() ** 2).sum().backward()
    assert rel_l2(eps.grad, e.grad) < TOL[dtype]


def test_2d_monitor_gradient_vs_oracle(cuda):
    shape, T = (40, 36), 120
    eps0 = _seeded(shape, 26)
    src = {"type": "gaussian_pulse", "row": 6}
    wl = [1500.0, 1550.0, 1600.0]
    e = eps0.clone().requires_grad_(True)
    o = R.run_2d(e, dl=15.0, dt=DT2(0.6, 15.0), omega=OMEGA, pml_layers=4, n_steps=T, source=src,
                 monitors=[dict(component="Ez", box=((30, 31), (0, 36)), wavelengths_nm=wl)])
    R.fom_abs2(o["monitors"][0]).backward()
    s = dn.FDTDSolver2D(grid_shape=shape, pml_layers=4, n_steps=T, dl=15.0, courant=0.6,
                        device=cuda, dtype=torch.float64)
    eps = eps0.clone().to(cuda).requires_grad_(True)
    r = s.forward(eps, source=dict(src),
                  monitors=[{"component": "Ez", "row": 30, "wavelengths_nm": wl}])
    (r.metadata["monitors"][0]["dft"].abs() ** 2).sum().backward()
    assert rel_l2(eps.grad, e.grad) < 1e-9


@pytest.mark.parametrize("pol,dtype", [("TM", torch.float32), ("TE", torch.float32),
                                       ("TM", torch.float64), ("TE", torch.float64)])
def test_adjoint2d_unaligned_rows_match_padded_rows(cuda, pol, dtype):
    """The 2-D reverse sweep through the C ABI with tight rows (pitch = W = 45:
    rows not on 16-byte boundaries, one value per lane) against the engine's
    padded rows (16-byte row access with a partly filled last lane): same
    adjoint fields and the same FP64 gradient."""
    import ctypes

    from diffnano_b200 import _lib
    from diffnano_b200.solvers import _setup
    from diffnano_b200.solvers._engine import Engine

    H, W, T = 38, 45, 30
    dl, courant = 20.0, 0.5
    dt = courant * dl / 2 ** 0.5
    src = {"type": "gaussian_pulse", "row": 9, "spread": 300.0, "t0": 400.0}
    p = _lib.DN_TM if pol == "TM" else _lib.DN_TE
    comp = _lib.DN_EZ if pol == "TM" else _lib.DN_HZ
    eng = Engine(is3d=False, shape=(H, W), dl=dl, dt=dt, pml_layers=6, dtype=dtype, device=cuda,
                 n_steps=T, wave=_setup.waveform_table(T, dt, OMEGA, src),
                 src_box=_setup.source_box_2d((H, W), src), src_comp=comp, pol=p)
    eng.set_eps(_seeded((H, W), 31))
    buf = eng.curl_buffer(T)
    rec = eng.curl_record(buf, 0, T)
    eng.run(0, T, record=rec)
    comps = (_lib.DN_EZ, _lib.DN_HX, _lib.DN_HY) if pol == "TM" else \
        (_lib.DN_HZ, _lib.DN_EX, _lib.DN_EY)
    g = torch.Generator().manual_seed(32)
    la = torch.zeros_like(eng.A)
    for c in comps:
        la[c, :, :, :W] = torch.randn(1, H, W, dtype=torch.float64, generator=g).to(cuda, dtype)
    la_t = la[..., :W].contiguous()
    lb = torch.zeros_like(la)
    grad = torch.zeros((1, H, eng.Wp), dtype=torch.float64, device=cuda)
    in_b = eng.adjoint(la, lb, rec, grad, None, 0, T, T)
    torch.cuda.synchronize(cuda)

    grid = type(eng.grid).from_buffer_copy(eng.grid)
    grid.pitch_y, grid.pitch_z = W, H * W
    lb_t = torch.zeros_like(la_t)
    ce_t = eng.ce[..., :W].contiguous()
    buf_t = buf[..., :W].contiguous()
    rec_t = _lib.DnCurlRecord(step_stride=H * W, t0=0, nslots=T)
    for n, c in enumerate(eng.eps_components()):
        rec_t.curl[c if c != _lib.DN_EZ else 2] = buf_t[n].data_ptr()
    grad_t = torch.zeros((1, H, W), dtype=torch.float64, device=cuda)
    assert (W * la_t.element_size()) % 16 != 0
    out = ctypes.c_int32(0)
    with torch.cuda.device(cuda):
        stream = torch.cuda.current_stream(cuda).cuda_stream
        rc = _lib.lib().dn_fdtd2d_adjoint(
            ctypes.byref(grid), _lib.PTR6(*[la_t[c].data_ptr() for c in range(6)]),
            _lib.PTR6(*[lb_t[c].data_ptr() for c in range(6)]), ce_t.data_ptr(),
            ctypes.byref(eng.cpml), ctypes.byref(rec_t), grad_t.data_ptr(), None, 0, T, T,
            eng.status.data_ptr(), ctypes.c_void_p(stream), ctypes.byref(out))
    assert rc == _lib.DN_OK
    eng.check_status()
    tol = 1e-6 if dtype == torch.float32 else 1e-13
    assert float(grad.abs().max()) > 0
    assert rel_l2(grad_t[0], grad[0, :, :W]) < tol
    res, res_t = (lb if in_b else la), (lb_t if out.value else la_t)
    for c in comps:
        assert rel_l2(res_t[c], res[c, :, :, :W]) < tol


def test_grad3d_central_finite_differences(cuda):
    """dL/deps at 16 seeded voxels vs central differences (h = 1e-3) of the
    FP64 kernels; L = sum |DFT Ey|^2 over a plane."""
    shape, T = (20, 20, 20), 80
    eps0 = _seeded(shape, 27)
    src = {"type": "gaussian_pulse", "plane": "xy", "z": 4, "component": "Ex",
           "spread": 400.0, "t0": 1200.0}
    mons = [{"component": "Ey", "plane": "xy", "z": 15, "extent": [[3, 17], [3, 17]],
             "wavelengths_nm": [1550.0]}]
    s = dn.FDTDSolver3D(grid_shape=shape, pml_layers=3, n_steps=T, device=cuda,
                        dtype=torch.float64)

    def loss(e):
        r = s.forward(e, source=dict(src), monitors=mons)
        return (r.metadata["monitors"][0]["dft"].abs() ** 2).sum()

    eps = eps0.clone().to(cuda).requires_grad_(True)
    loss(eps).backward()
    gen = torch.Generator().manual_seed(28)
    idx = torch.randint(3, 17, (16, 3), generator=gen)
    h = 1e-3
    fd, ad = [], []
    with torch.no_grad():
        for z, y, x in idx.tolist():
            ep = eps0.clone().to(cuda)
            ep[z, y, x] += h
            em = eps0.clone().to(cuda)
            em[z, y, x] -= h
            fd.append((loss(ep) - loss(em)).item() / (2 * h))
            ad.append(eps.grad[z, y, x].item())
    assert rel_l2(torch.tensor(ad), torch.tensor(fd)) < 1e-4


def test_fom_kernel_matches_torch_and_is_deterministic(cuda):
    from diffnano_b200.solvers import fom_abs2

    g = torch.Generator().manual_seed(30)
    for n in (1, 31, 4096, 300_001):
        z = torch.complex(torch.randn(n, dtype=torch.float64, generator=g),
                          torch.randn(n, dtype=torch.float64, generator=g)).to(cuda)
        a = fom_abs2(z)
        b = fom_abs2(z)
        ref = (z.abs() ** 2).sum()
        assert torch.equal(a, b)
        assert abs(float(a) - float(ref)) <= 1e-12 * float(ref)


def test_fom_kernel_gradient_drives_the_adjoint(cuda):
    """The FOM kernel's backward feeds the monitor adjoint like torch's |F|^2."""
    from diffnano_b200.solvers import fom_abs2

    shape, T = (16, 16, 16), 40
    eps0 = _seeded(shape, 31)
    src = {"type": "gaussian_pulse", "plane": "xy", "z": 4, "component": "Ex",
           "spread": 300.0, "t0": 900.0}
    mons = [{"component": "Ey", "plane": "xy", "z": 12, "wavelengths_nm": [1550.0]}]
    s = dn.FDTDSolver3D(grid_shape=shape, pml_layers=3, n_steps=T, device=cuda,
                        dtype=torch.float64)
    grads = []
    for use_kernel in (True, False):
        eps = eps0.clone().to(cuda).requires_grad_(True)
        F = s.forward(eps, source=dict(src), monitors=mons).metadata["monitors"][0]["dft"]
        (fom_abs2(F) if use_kernel else (F.abs() ** 2).sum()).backward()
        grads.append(eps.grad)
    assert rel_l2(grads[0], grads[1]) < 1e-12
