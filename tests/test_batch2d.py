"""Batched 2-D path (one persistent launch for many grids) against the
single-grid solver: fields, monitor DFTs and dL/deps of every instance, with
ragged sizes, different step counts, several checkpoint segments, TM and TE,
every tile height, and the CUDA-graph replay."""

from __future__ import annotations

import pytest
import torch
from conftest import rel_l2

import diffnano_b200 as dn
from diffnano_b200 import _lib
from diffnano_b200.solvers.batch2d import BatchInstance, FDTDBatch2D, autotune_tile_rows

pytestmark = pytest.mark.gpu

SHAPES = [(40, 36), (70, 50), (33, 90), (64, 64), (20, 24)]
STEPS = [60, 45, 90, 30, 75]


def _specs(pol, monitor=True):
    out = []
    for n, (shape, T) in enumerate(zip(SHAPES, STEPS)):
        src = {"type": "gaussian_pulse", "row": 5 + n, "spread": 300.0, "t0": 900.0}
        mon = {"row": shape[0] - 6, "wavelengths_nm": [1500.0, 1550.0 + 20 * n]} if monitor else None
        out.append(BatchInstance(grid_shape=shape, n_steps=T, dl=20.0,
                                 wavelength_nm=1450.0 + 40 * n, pml_layers=4, courant=0.5,
                                 source=src, monitor=mon))
    return out


def _eps(seed):
    g = torch.Generator().manual_seed(seed)
    return [1.5 + 2.0 * torch.rand(*s, dtype=torch.float64, generator=g) for s in SHAPES]


def _single(spec, pol, dtype, cuda, eps):
    s = dn.FDTDSolver2D(grid_shape=spec.grid_shape, dl=spec.dl, wavelength_nm=spec.wavelength_nm,
                        polarization=pol, pml_layers=spec.pml_layers, n_steps=spec.n_steps,
                        courant=spec.courant, device=cuda, dtype=dtype)
    comp = "Ez" if pol == "TM" else "Hz"
    mons = [{"component": comp, **spec.monitor}] if spec.monitor else None
    return s.forward(eps, source=dict(spec.source), monitors=mons)


@pytest.mark.parametrize("rows", [8, 16, 32])
@pytest.mark.parametrize("pol", ["TM", "TE"])
def test_batched_forward_matches_single_grids(cuda, pol, rows):
    specs = _specs(pol)
    eps = _eps(1)
    b = FDTDBatch2D(specs, pol, torch.float32, cuda, checkpoint_interval=16, tile_rows=rows)
    fields, dfts = b.forward([e.to(cuda) for e in eps])
    for spec, e, f, d in zip(specs, eps, fields, dfts):
        r = _single(spec, pol, torch.float32, cuda, e.to(cuda))
        assert rel_l2(f, r.field[0]) < 1e-6
        assert rel_l2(torch.view_as_real(d), torch.view_as_real(r.metadata["monitors"][0]["dft"])) < 1e-6


@pytest.mark.parametrize("rows", [8, 16, 32])
@pytest.mark.parametrize("pol", ["TM", "TE"])
def test_batched_gradients_match_single_grids(cuda, pol, rows):
    """Every tile height: 1, 2 or 4 rows per warp (a one-row warp owns no
    neighbouring row of its reverse sweep)."""
    specs = _specs(pol)
    eps0 = _eps(2)
    gen = torch.Generator().manual_seed(3)
    G = [torch.randn(*s, dtype=torch.float64, generator=gen) for s in SHAPES]
    b = FDTDBatch2D(specs, pol, torch.float64, cuda, checkpoint_interval=7, tile_rows=rows)
    eps = [e.clone().to(cuda).requires_grad_(True) for e in eps0]
    fields, dfts = b.forward(eps)
    loss = sum((f * g.to(cuda)).sum() + (d.abs() ** 2).sum() for f, g, d in zip(fields, G, dfts))
    loss.backward()
    for spec, e0, e, g in zip(specs, eps0, eps, G):
        ref = e0.clone().to(cuda).requires_grad_(True)
        r = _single(spec, pol, torch.float64, cuda, ref)
        ((r.field[0] * g.to(cuda)).sum() + (r.metadata["monitors"][0]["dft"].abs() ** 2).sum()).backward()
        assert rel_l2(e.grad, ref.grad) < 1e-9


def test_batched_graph_replay_matches_direct(cuda):
    specs = _specs("TM")
    b = FDTDBatch2D(specs, "TM", torch.float32, cuda, tile_rows=16)
    for seed in (4, 5):
        eps = [e.to(cuda) for e in _eps(seed)]
        f_graph, d_graph = b.forward_graphed(eps)
        f_direct, d_direct = b.run_forward(eps)
        for a, c in zip(f_graph, f_direct):
            assert torch.equal(a, c)


def test_autotuner_picks_a_candidate_and_caches(cuda, tmp_path, monkeypatch):
    monkeypatch.setenv("XDG_CACHE_HOME", str(tmp_path))
    b = FDTDBatch2D(_specs("TM", monitor=False), "TM", torch.float32, cuda)
    rows = autotune_tile_rows(b)
    assert rows in (8, 16, 32)
    assert (tmp_path / "diffnano_b200" / "autotune.json").exists()
    assert autotune_tile_rows(b) == rows


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("pol", ["TM", "TE"])
def test_cluster_forward_matches_persistent_kernel(cuda, pol, dtype):
    """Gradient-free solves keep each grid in one thread-block cluster's shared
    memory; same fields and DFTs as the tile-by-tile persistent kernel.  The
    large instances (400 x 320 FP32, 386 x 97 FP64) fill most of a cluster's
    shared memory and have row bands that do not divide the height."""
    big = (400, 320) if dtype == torch.float32 else (386, 97)
    shapes = SHAPES + [big]
    specs = _specs(pol) + [BatchInstance(grid_shape=big, n_steps=50, dl=20.0,
                                         pml_layers=6, courant=0.5,
                                         source={"type": "gaussian_pulse", "row": 9,
                                                 "spread": 300.0, "t0": 900.0},
                                         monitor={"col": 40, "wavelengths_nm": [1550.0]})]
    g = torch.Generator().manual_seed(3)
    eps = [(1.5 + 2.0 * torch.rand(*s, dtype=torch.float64, generator=g)).to(cuda)
           for s in shapes]
    a = FDTDBatch2D(specs, pol, dtype, cuda, tile_rows=16, cluster=True)
    b = FDTDBatch2D(specs, pol, dtype, cuda, tile_rows=16, cluster=False)
    fa, da = a.forward(eps)
    fb, db = b.forward(eps)
    a.check_status()
    b.check_status()
    assert a.uses_cluster(False) and not b.uses_cluster(False) and not a.uses_cluster(True)
    # both large grids fit twice: the double-buffered kernel, one barrier per step
    assert a._cluster[0] == 16 | _lib.DN_CLUSTER_DOUBLE_BUFFERED
    tol = 1e-6 if dtype == torch.float32 else 1e-13
    for x, y in zip(fa, fb):
        assert rel_l2(x, y) < tol
    for x, y in zip(da, db):
        assert rel_l2(torch.view_as_real(x), torch.view_as_real(y)) < tol
    # graph replay uses the cluster kernel too
    fg, dg = a.forward_graphed(eps)
    for x, y in zip(fg, fa):
        assert torch.equal(x, y)


@pytest.mark.gpu
@pytest.mark.parametrize("pol", ["TM", "TE"])
def test_cluster_in_place_kernel_for_grids_that_fit_once(cuda, pol):
    """A 460 x 400 FP32 grid fits a 16-CTA cluster's shared memory once but not
    twice: the in-place cluster kernel (two barriers per step) runs it, with the
    tile kernel's fields and DFTs."""
    spec = BatchInstance(grid_shape=(460, 400), n_steps=40, dl=20.0, pml_layers=6, courant=0.5,
                         source={"type": "gaussian_pulse", "row": 9, "spread": 300.0,
                                 "t0": 900.0},
                         monitor={"col": 40, "wavelengths_nm": [1550.0]})
    g = torch.Generator().manual_seed(5)
    eps = [(1.5 + 2.0 * torch.rand(460, 400, dtype=torch.float64, generator=g)).to(cuda)]
    a = FDTDBatch2D([spec], pol, torch.float32, cuda, tile_rows=16, cluster=True)
    b = FDTDBatch2D([spec], pol, torch.float32, cuda, tile_rows=16, cluster=False)
    fa, da = a.forward(eps)
    fb, db = b.forward(eps)
    a.check_status()
    b.check_status()
    assert a.uses_cluster(False) and a._cluster[0] == 16  # packed on the first forward
    for x, y in zip(fa, fb):
        assert rel_l2(x, y) < 1e-6
    for x, y in zip(da, db):
        assert rel_l2(torch.view_as_real(x), torch.view_as_real(y)) < 1e-6


def test_grid_barrier_wait_runs_out_and_reports_timeout(cuda):
    """The persistent kernels' grid barrier (dn_batch2d_barrier_selftest runs it
    alone): all arrivals -> DN_OK; one arrival that never comes -> every CTA's
    bounded wait runs out, the status reads DN_ETIMEOUT within milliseconds,
    and the context stays usable: a persistent batched solve after it gives
    the same fields as one before it."""
    import ctypes
    import time

    L = _lib.lib()
    specs = _specs("TM")
    eps = [e.to(cuda) for e in _eps(7)]
    b = FDTDBatch2D(specs, "TM", torch.float32, cuda, tile_rows=16, cluster=False)
    before, _ = b.forward(eps)
    b.check_status()
    bar = torch.zeros(4, dtype=torch.int32, device=cuda)
    st = torch.zeros(1, dtype=torch.int32, device=cuda)
    stream = ctypes.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    rc = L.dn_batch2d_barrier_selftest(8, 0, 1 << 16, 200, bar.data_ptr(), st.data_ptr(), stream)
    torch.cuda.synchronize(cuda)
    assert rc == _lib.DN_OK and int(st.item()) == _lib.DN_OK
    t0 = time.perf_counter()
    rc = L.dn_batch2d_barrier_selftest(8, 1, 1 << 12, 3, bar.data_ptr(), st.data_ptr(), stream)
    torch.cuda.synchronize(cuda)
    elapsed = time.perf_counter() - t0
    assert rc == _lib.DN_OK and int(st.item()) == _lib.DN_ETIMEOUT
    assert elapsed < 5.0
    after, _ = b.forward(eps)
    b.check_status()
    for x, y in zip(before, after):
        assert torch.equal(x, y)


@pytest.mark.parametrize("pol", ["TM", "TE"])
def test_uniform_batch_keeps_batch_wide_storage_and_matches_single_grids(cuda, pol):
    """Instances with one grid, step count, time step and monitor share
    batch-wide field / coefficient / monitor tensors (one-op upload, reset
    and outputs); fields, DFTs and gradients still match single-grid solves."""
    shape = (44, 40)
    spec = BatchInstance(grid_shape=shape, n_steps=50, dl=20.0, wavelength_nm=1550.0,
                         pml_layers=4, courant=0.5,
                         source={"type": "gaussian_pulse", "row": 6, "spread": 300.0,
                                 "t0": 900.0},
                         monitor={"row": 36, "wavelengths_nm": [1500.0, 1600.0]})
    specs = [spec] * 4
    gen = torch.Generator().manual_seed(9)
    eps0 = [1.5 + 2.0 * torch.rand(*shape, dtype=torch.float64, generator=gen) for _ in specs]
    G = [torch.randn(*shape, dtype=torch.float64, generator=gen) for _ in specs]
    b = FDTDBatch2D(specs, pol, torch.float64, cuda, checkpoint_interval=7, tile_rows=16,
                    cluster=False)
    eps = [e.clone().to(cuda).requires_grad_(True) for e in eps0]
    fields, dfts = b.forward(eps)
    assert b._stack is not None
    loss = sum((f * g.to(cuda)).sum() + (d.abs() ** 2).sum() for f, g, d in zip(fields, G, dfts))
    loss.backward()
    for e0, e, f, d, g in zip(eps0, eps, fields, dfts, G):
        ref = e0.clone().to(cuda).requires_grad_(True)
        r = _single(spec, pol, torch.float64, cuda, ref)
        assert rel_l2(f, r.field[0]) < 1e-12
        dr = r.metadata["monitors"][0]["dft"]
        assert rel_l2(torch.view_as_real(d), torch.view_as_real(dr)) < 1e-11
        ((r.field[0] * g.to(cuda)).sum() + (dr.abs() ** 2).sum()).backward()
        assert rel_l2(e.grad, ref.grad) < 1e-9


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_graphed_fom_gradient_matches_autograd(cuda, dtype):
    """Forward, adjoint seeding and backward of every instance recorded in one
    CUDA graph: FOM = sum |DFT|^2 and dFOM/deps equal the autograd path's;
    replays with new eps recompute, a replay with the first eps again
    reproduces the first results bit for bit."""
    specs = _specs("TM")
    eps_a, eps_b = _eps(11), _eps(12)
    b = FDTDBatch2D(specs, "TM", dtype, cuda, checkpoint_interval=16, tile_rows=16)
    fom, grads = b.fom_gradient_graphed([e.to(cuda) for e in eps_a])
    fom_a, grads_a = fom.clone(), [g.clone() for g in grads]
    fom, grads = b.fom_gradient_graphed([e.to(cuda) for e in eps_b])
    fom_b = fom.clone()
    assert not torch.equal(fom_a, fom_b)
    fom, grads = b.fom_gradient_graphed([e.to(cuda) for e in eps_a])
    assert torch.equal(fom, fom_a) and all(torch.equal(x, y) for x, y in zip(grads, grads_a))
    ref = FDTDBatch2D(specs, "TM", dtype, cuda, checkpoint_interval=16, tile_rows=16)
    e_dev = [e.to(cuda).requires_grad_(True) for e in eps_a]
    _, dfts = ref.forward(e_dev)
    foms = torch.stack([(torch.view_as_real(d.to(torch.complex128)) ** 2).sum() for d in dfts])
    foms.sum().backward()
    assert rel_l2(fom_a, foms.detach()) < 1e-14
    for g, e in zip(grads_a, e_dev):
        assert rel_l2(g, e.grad) < 1e-12
