"""Non-finite watchdog on the GPU.

The reference's TE update grows exponentially (``fdtd2d.py:269-303``): the
300-step fixture reaches ~2e87 in FP64, far beyond FP32's range, so an FP32
run overflows to Inf/NaN.  The reference returns such fields silently; here
every solver path scans its outputs once per solve and raises DN_ENONFINITE.
The overflow is numerical (ordinary IEEE arithmetic in the kernels), not a
device fault.
"""

from __future__ import annotations

import pytest
import torch
from conftest import load_golden, rel_l2

import diffnano_b200 as dn
from diffnano_b200 import _lib

pytestmark = pytest.mark.gpu


def _te_long(cuda, dtype):
    g = load_golden("te2d_long")
    s = dn.FDTDSolver2D(grid_shape=(48, 40), polarization="TE", pml_layers=6,
                        n_steps=int(g["n_steps"]), device=cuda, dtype=dtype)
    return g, s


def test_fp32_te_overflow_raises_on_every_path(cuda):
    g, s = _te_long(cuda, torch.float32)
    eps = torch.tensor(g["eps"]).to(cuda)
    # gradient-free: whole grid in one thread-block cluster
    with pytest.raises(_lib.DNError) as e1:
        s.forward(eps, source=dict(g["source"]))
    assert e1.value.status == _lib.DN_ENONFINITE
    # with a gradient: per-step kernels and checkpoints (raises in the forward)
    e = eps.clone().requires_grad_(True)
    with pytest.raises(_lib.DNError) as e2:
        s.forward(e, source=dict(g["source"]))
    assert e2.value.status == _lib.DN_ENONFINITE
    # the probe series path (time_series)
    with pytest.raises(_lib.DNError) as e3:
        s.time_series(eps, probe=(20, 20), source=dict(g["source"]))
    assert e3.value.status == _lib.DN_ENONFINITE


def test_fp64_te_long_stays_finite_and_a_solver_recovers(cuda):
    g, s = _te_long(cuda, torch.float64)
    r = s.forward(torch.tensor(g["eps"]).to(cuda), source=dict(g["source"]))
    assert rel_l2(r.field[0], g["hz"]) < 1e-12
    # after an FP32 overflow the same kind of solver runs a finite problem cleanly
    g2 = load_golden("te2d")
    s32 = dn.FDTDSolver2D(grid_shape=(48, 40), polarization="TE", pml_layers=6,
                          n_steps=int(g["n_steps"]), device=cuda, dtype=torch.float32)
    with pytest.raises(_lib.DNError):
        s32.forward(torch.tensor(g["eps"]).to(cuda), source=dict(g["source"]))
    s32.n_steps = int(g2["n_steps"])
    r2 = s32.forward(torch.tensor(g2["eps"]).to(cuda), source=dict(g2["source"]))
    assert rel_l2(r2.field[0], g2["hz"]) < 1e-5


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("bad", [float("nan"), float("inf"), float("-inf")])
def test_check_finite_kernel_finds_one_bad_value(cuda, dtype, bad):
    """One bad element anywhere in several strided arrays is found; clean
    arrays leave the status word at DN_OK."""
    gen = torch.Generator(device=cuda).manual_seed(3)
    padded = torch.randn(6, 9, 33, 64, dtype=dtype, device=cuda, generator=gen)
    flat = torch.randn(5000, dtype=dtype, device=cuda, generator=gen)
    views = [padded[c, :, :, :50] for c in range(6)] + [flat]
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    stream = torch.cuda.current_stream(cuda).cuda_stream
    _lib.check_finite(views, status, stream)
    assert int(status.item()) == _lib.DN_OK
    # padding columns are outside every span: a NaN there is not reported
    padded[2, 4, 7, 60] = float("nan")
    _lib.check_finite(views, status, stream)
    assert int(status.item()) == _lib.DN_OK
    for where in [(0, 0, 0, 0), (5, 8, 32, 49), (3, 4, 17, 25)]:
        status.zero_()
        saved = float(padded[where])
        padded[where] = bad
        _lib.check_finite(views, status, stream)
        assert int(status.item()) == _lib.DN_ENONFINITE, where
        padded[where] = saved
    status.zero_()
    flat[4999] = bad
    _lib.check_finite(views, status, stream)
    assert int(status.item()) == _lib.DN_ENONFINITE
