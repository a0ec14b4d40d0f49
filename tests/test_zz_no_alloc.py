"""dn_fdtd2d_run_noalloc: the 2-D step run for callers that cannot allocate
device memory where they step the solver (a plugin inside an application that
owns the whole device-memory budget, or a loop whose policy forbids
allocation).  It uses a fixed device array in the library as the second half
of the ping-pong pair instead of a caller-provided second field set.

Checked through the C ABI against the allocating entry point
(dn_fdtd2d_run), on two calls in a row (an odd step count, which leaves the
result in the library's array and copies it back, then an even one), and
the size limit.  This file is collected last on purpose (its name sorts
after the other test files) and holds no state between tests, so it passes
alone in a fresh process and after the rest of the suite.
"""

from __future__ import annotations

import ctypes

import pytest
import torch
from conftest import rel_l2

from diffnano_b200 import _lib
from diffnano_b200.solvers import _setup
from diffnano_b200.solvers._engine import Engine

pytestmark = pytest.mark.gpu

TOL = {torch.float32: 1e-5, torch.float64: 1e-12}


def _engine(shape, pol, dtype, dev, n_steps):
    src = {"type": "gaussian_pulse", "row": 9, "spread": 500.0, "t0": 1500.0}
    dl, courant = 20.0, 0.5
    dt = courant * dl / 2 ** 0.5
    omega = 2 * 3.141592653589793 / 1550.0
    comp = _lib.DN_EZ if pol == _lib.DN_TM else _lib.DN_HZ
    eng = Engine(is3d=False, shape=shape, dl=dl, dt=dt, pml_layers=6, dtype=dtype, device=dev,
                 n_steps=n_steps, wave=_setup.waveform_table(n_steps, dt, omega, src),
                 src_box=_setup.source_box_2d(shape, src), src_comp=comp, pol=pol)
    g = torch.Generator().manual_seed(3)
    eng.set_eps(1.5 + 2.0 * torch.rand(*shape, dtype=torch.float64, generator=g))
    return eng


def _noalloc(eng, F, t0, n):
    L = _lib.lib()
    with torch.cuda.device(eng.device):
        stream = torch.cuda.current_stream(eng.device).cuda_stream
        return L.dn_fdtd2d_run_noalloc(
            ctypes.byref(eng.grid), _lib.PTR6(*[F[c].data_ptr() for c in range(6)]),
            eng.ce.data_ptr(), ctypes.byref(eng.cpml), ctypes.byref(eng.src), None, 0, None,
            int(t0), int(n), eng.status.data_ptr(), ctypes.c_void_p(stream))


@pytest.mark.parametrize("pol,dtype", [(_lib.DN_TM, torch.float32), (_lib.DN_TE, torch.float64)])
def test_noalloc_matches_allocating_entry_point_on_two_calls(cuda, pol, dtype):
    shape = (96, 80)
    steps = (7, 6)
    eng = _engine(shape, pol, dtype, cuda, sum(steps))
    F = torch.zeros_like(eng.A)  # the caller's only field set
    comps = (_lib.DN_EZ, _lib.DN_HX, _lib.DN_HY) if pol == _lib.DN_TM else \
        (_lib.DN_HZ, _lib.DN_EX, _lib.DN_EY)
    t0 = 0
    for n in steps:
        eng.run(t0, n)  # allocating path: caller-owned ping-pong pair A/B
        rc = _noalloc(eng, F, t0, n)
        assert rc == _lib.DN_OK, _lib.lib().dn_strerror(rc)
        torch.cuda.synchronize(cuda)
        t0 += n
        W = shape[1]
        for c in comps:
            ref = eng.field(c)
            got = F[c, :, :, :W]
            assert float(ref.abs().max()) > 0
            assert rel_l2(got, ref) < TOL[dtype]
    eng.check_status()


def test_noalloc_rejects_grids_beyond_its_array(cuda):
    shape = (1024, 1024)  # 3 x 4 MiB of FP32 fields > the 6 MiB array
    eng = _engine(shape, _lib.DN_TM, torch.float32, cuda, 2)
    F = torch.zeros_like(eng.A)
    assert _noalloc(eng, F, 0, 1) == _lib.DN_ENOMEM
    assert 3 * 1024 * eng.Wp * 4 > _lib.DN_NOALLOC_MAX_BYTES
