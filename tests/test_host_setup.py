"""Host-side set-up (no GPU): waveform tables, CPML profiles, source boxes,
monitor specs and the solver API surface, checked against the oracle and the
reference's golden outputs."""

from __future__ import annotations

import json
import math

import numpy as np
import pytest
import torch
from conftest import DT2, DT3, OMEGA, load_golden

import diffnano_b200 as dn
from diffnano_b200.solvers import Solver, _setup
from diffnano_b200.solvers._common import GridShapeError, checkpoint_interval
from oracle import fdtd_ref as R


@pytest.mark.parametrize("name,courant,dl,T", [("tm2d_cfg0", 0.5, 20.0, 2000),
                                               ("te2d", 0.5, 20.0, 40),
                                               ("te2d_long", 0.5, 20.0, 300),
                                               ("tm2d_cont", 0.6, 15.0, 250)])
def test_waveform_table_matches_reference(name, courant, dl, T):
    g = load_golden(name)
    w = _setup.waveform_table(T, DT2(courant, dl), OMEGA, g["source"]).numpy()
    # vectorised FP32 sine vs the reference's scalar one: equal to ~1 FP32 ulp
    np.testing.assert_allclose(w, g["wave"], rtol=0, atol=2 ** -23 * np.abs(g["wave"]).max())


def test_waveform_unknown_type_is_zero():
    assert float(_setup.waveform_table(10, 1.0, 0.1, {"type": "nope"}).abs().sum()) == 0.0


@pytest.mark.parametrize("n,L,dl,dt", [(256, 20, 20.0, DT2(0.5, 20.0)), (37, 5, 25.0, DT3(0.4, 25.0)),
                                       (10, 0, 20.0, 1.0), (6, 4, 20.0, 3.0)])
def test_cpml_profile_matches_oracle(n, L, dl, dt):
    b, c = _setup.cpml_profile(n, L, dl, dt)
    rb, rc = R.cpml_profile(n, L, dl, dt)
    assert torch.equal(b, rb) and torch.equal(c, rc)


@pytest.mark.parametrize("src", [{}, {"pos": [3, 4]}, {"pos": [99, 0]}, {"row": 2}, {"row": -1}])
def test_source_box_2d_matches_oracle(src):
    shape = (12, 10)
    ob = R.source_box_2d(shape, src)
    b = _setup.source_box_2d(shape, src)
    assert (ob is None) == (b is None)
    if b is not None:
        assert b[1:] == ob


@pytest.mark.parametrize("src", [{}, {"pos": [1, 2, 3]}, {"pos": [1, 2, 30]},
                                 {"plane": "xy", "z": 3}, {"plane": "xz"}, {"plane": "yz", "x": 9},
                                 {"plane": "yz", "x": 99}])
def test_source_box_3d_matches_oracle(src):
    shape = (8, 9, 10)
    assert _setup.source_box_3d(shape, src) == R.source_box_3d(shape, src)


def test_monitor_boxes_and_validation():
    assert _setup.monitor_box({"row": 5}, (1, 10, 12), False) == ((0, 1), (5, 6), (0, 12))
    assert _setup.monitor_box({"col": 2}, (1, 10, 12), False) == ((0, 1), (0, 10), (2, 3))
    assert _setup.monitor_box({"plane": "xy", "z": 4, "extent": [[2, 6], [3, 9]]},
                              (8, 10, 12), True) == ((4, 5), (2, 6), (3, 9))
    with pytest.raises(ValueError):
        _setup.monitor_box({"row": 10}, (1, 10, 12), False)
    with pytest.raises(ValueError):
        _setup.monitor_box({"plane": "qq"}, (8, 10, 12), True)


def test_dft_phase_table_matches_oracle():
    ph = _setup.dft_phase_table(50, 7.0, [1500.0, 1550.0])
    ref = R.dft_phase(50, 7.0, [1500.0, 1550.0])
    assert float((ph - ref).abs().max()) < 1e-13


def test_solver_api_surface():
    s2 = dn.FDTDSolver2D(grid_shape=(20, 20), pml_layers=0, n_steps=10)
    assert s2.grid_shape == (20, 20) and s2.n_steps == 10 and s2.courant == 0.5
    assert math.isclose(s2.dt, 0.5 * 20.0 / math.sqrt(2.0))
    assert isinstance(s2, Solver)
    s3 = dn.FDTDSolver3D(grid_shape=(10, 10, 10), pml_layers=0, n_steps=5)
    assert s3.courant == 0.4 and isinstance(s3, Solver)
    assert s3.device == torch.device("cpu")
    m = s3._build_source_mask({"plane": "xy", "z": 3})
    assert float(m.sum()) == 100.0 and float(m[3].sum()) == 100.0
    assert float(s2._build_source_mask({"pos": [50, 50]}).sum()) == 0.0


def test_non_cubic_reference_axes_rejected_and_physical_accepted():
    s = dn.FDTDSolver3D(grid_shape=(8, 8, 16))
    with pytest.raises(GridShapeError):
        s._axes()
    with pytest.raises(RuntimeError):  # the reference raises RuntimeError here
        s._axes()
    assert dn.FDTDSolver3D(grid_shape=(8, 8, 16), cpml_axes="physical")._axes() == 1


def test_no_cpu_path():
    if torch.cuda.is_available():
        pytest.skip("has a GPU")
    with pytest.raises(RuntimeError, match="no CPU path"):
        dn.FDTDSolver2D(grid_shape=(8, 8), n_steps=2).forward(torch.ones(8, 8))


def test_checkpoint_interval():
    assert checkpoint_interval(4000, False, 4) == 64
    assert checkpoint_interval(10, True, 2) == 5
    assert checkpoint_interval(1, False, 4) == 1


def test_2d_engine_reuse_decisions():
    """FDTDSolver2D._engine_for on the host (engine construction stubbed):
    one engine per gradient-free set-up, reused; a fresh one per gradient
    call; no caching of set-ups that are not plain JSON; at most four kept."""
    s = dn.FDTDSolver2D(grid_shape=(16, 16), n_steps=5)
    made = []

    def fake(n_steps, src, mons, probe=None):
        made.append((n_steps, json.dumps(src, default=str), probe))
        return object()

    s._make_engine = fake
    src_a = {"type": "gaussian_pulse", "row": 3}
    src_b = {"type": "gaussian_pulse", "row": 4}
    e1 = s._engine_for(src_a, None, None, reuse=True)
    assert s._engine_for(dict(src_a), None, None, reuse=True) is e1
    assert s._engine_for(src_b, None, None, reuse=True) is not e1
    assert s._engine_for(src_a, None, None, reuse=False) is not e1  # gradient call
    assert len(made) == 3
    # a tensor in the source dict: built every time, never cached
    src_t = {"type": "gaussian_pulse", "row": 3, "amplitude": torch.tensor(2.0)}
    assert s._engine_for(src_t, None, None, reuse=True) is not s._engine_for(src_t, None, None,
                                                                               reuse=True)
    assert len(s._engine_cache) == 2
    for r in range(5, 9):
        s._engine_for({"type": "gaussian_pulse", "row": r}, None, None, reuse=True)
    assert len(s._engine_cache) <= 4


def test_batch_wide_storage_decision():
    """FDTDBatch2D._stacked_views on the host (CPU tensors): identical
    instances get views of one batch-wide tensor per array; any difference
    in grid, steps or monitor keeps per-instance storage."""
    from diffnano_b200.solvers.batch2d import BatchInstance, FDTDBatch2D

    def spec(shape=(20, 24), T=30, mon=True):
        return BatchInstance(grid_shape=shape, n_steps=T, dl=20.0, pml_layers=4, courant=0.5,
                             source={"type": "gaussian_pulse", "row": 5},
                             monitor={"row": 12, "wavelengths_nm": [1500.0, 1600.0]} if mon
                             else None)

    def views(specs):
        b = FDTDBatch2D.__new__(FDTDBatch2D)
        b.specs, b.dtype, b.device = specs, torch.float32, torch.device("cpu")
        return b, b._stacked_views()

    b, v = views([spec()] * 3)
    assert v is not None and len(v) == 3
    f, ce, acc = b._stack
    assert f.shape == (3, 2, 3, 20, 32) and ce.shape == (3, 20, 32) and acc.shape == (3, 2, 24, 2)
    assert v[1][0].data_ptr() == f.data_ptr() + f[0].numel() * f.element_size()
    assert v[2][2].shape == (2, 24, 2)
    for other in (spec(shape=(20, 28)), spec(T=31), spec(mon=False)):
        b, v = views([spec(), spec(), other])
        assert v is None and b._stack is None
    b, v = views([spec(mon=False)] * 2)
    assert v is not None and b._stack[2] is None and v[0][2] is None
    b, v = views([spec()])
    assert v is None
