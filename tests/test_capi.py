"""The C-ABI library loads and exports every symbol include/*.h declares;
argument validation rejects bad calls on the host (no GPU work)."""

from __future__ import annotations

import ctypes
import glob
import os
import re

import pytest
from conftest import ROOT

from diffnano_b200 import _lib


def _declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(dn_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    declared = _declared_symbols()
    assert "dn_fdtd3d_run" in declared and "dn_fdtd2d_run" in declared
    for name in declared:
        assert hasattr(L, name), f"{name} declared in include/ but not exported"
    assert set(declared) <= set(_lib.SIGNATURES), "ctypes signatures missing for some symbols"


def test_strerror_and_version():
    L = _lib.lib()
    assert L.dn_version() >= 1
    assert L.dn_strerror(_lib.DN_OK) == b"ok"
    assert L.dn_strerror(_lib.DN_ETIMEOUT).startswith(b"bounded")
    assert L.dn_strerror(12345) == b"unknown status"


@pytest.mark.parametrize("fn", ["dn_fdtd2d_run", "dn_fdtd3d_run"])
def test_null_grid_rejected(fn):
    L = _lib.lib()
    out = ctypes.c_int32(-1)
    rc = getattr(L, fn)(None, None, None, None, None, None, None, 0, None, None, 0, 1, None, None,
                        ctypes.byref(out))
    assert rc == _lib.DN_EINVAL


def _grid(**kw):
    g = dict(D=1, H=8, W=8, dtype=_lib.DN_F32, pitch_y=32, pitch_z=256, dt=1.0, dl=2.0, axes=0,
             pol=0)
    g.update(kw)
    return _lib.DnGrid(**g)


@pytest.mark.parametrize("bad", [dict(H=0), dict(pitch_y=4), dict(dt=0.0), dict(dl=-1.0),
                                 dict(dtype=7), dict(pol=9), dict(D=2)])
def test_2d_bad_grid_rejected_before_any_launch(bad):
    L = _lib.lib()
    g = _grid(**bad)
    fake = _lib.PTR6(*([16] * 6))  # never dereferenced: validation fails first
    cp = _lib.DnCpml()
    for a in range(3):
        cp.b[a] = cp.c[a] = 16
    out = ctypes.c_int32(-1)
    rc = L.dn_fdtd2d_run(ctypes.byref(g), fake, fake, 16, ctypes.byref(cp), None, None, 0, None,
                         None, 0, 1, None, None, ctypes.byref(out))
    assert rc == _lib.DN_EINVAL


def test_3d_reference_axes_needs_cubic_grid():
    L = _lib.lib()
    g = _grid(D=4, H=8, W=8, pitch_z=256, axes=_lib.DN_AXES_REFERENCE)
    fake = _lib.PTR6(*([256] * 6))
    cp = _lib.DnCpml()
    for a in range(3):
        cp.b[a] = cp.c[a] = 256
    out = ctypes.c_int32(-1)
    rc = L.dn_fdtd3d_run(ctypes.byref(g), fake, fake, 256, ctypes.byref(cp), None, None, 0,
                         None, None, 0, 1, None, None, ctypes.byref(out))
    assert rc == _lib.DN_EINVAL


def test_source_box_outside_grid_rejected():
    L = _lib.lib()
    g = _grid()
    fake = _lib.PTR6(*([16] * 6))
    cp = _lib.DnCpml()
    for a in range(3):
        cp.b[a] = cp.c[a] = 16
    src = _lib.DnSource(component=_lib.DN_EZ, box=_lib.box((0, 0, 0), (1, 9, 8)), wave=16)
    out = ctypes.c_int32(-1)
    rc = L.dn_fdtd2d_run(ctypes.byref(g), fake, fake, 16, ctypes.byref(cp), ctypes.byref(src),
                         None, 0, None, None, 0, 1, None, None, ctypes.byref(out))
    assert rc == _lib.DN_EINVAL
    # a TE-only component on a TM grid is rejected too
    src = _lib.DnSource(component=_lib.DN_HZ, box=_lib.box((0, 0, 0), (1, 1, 1)), wave=16)
    rc = L.dn_fdtd2d_run(ctypes.byref(g), fake, fake, 16, ctypes.byref(cp), ctypes.byref(src),
                         None, 0, None, None, 0, 1, None, None, ctypes.byref(out))
    assert rc == _lib.DN_EINVAL


def test_check_maps_status_to_exceptions():
    with pytest.raises(ValueError):
        _lib.check("x", _lib.DN_EINVAL)
    with pytest.raises(_lib.DNError):
        _lib.check("x", _lib.DN_ETIMEOUT)
    _lib.check("x", _lib.DN_OK)


@pytest.mark.parametrize("fn", ["dn_fdtd2d_adjoint", "dn_fdtd3d_adjoint"])
def test_adjoint_rejects_missing_curl_record(fn):
    L = _lib.lib()
    is3d = fn.startswith("dn_fdtd3d")
    g = _grid(D=8 if is3d else 1, H=8, W=8, pitch_y=32, pitch_z=256)
    fake = _lib.PTR6(*([256] * 6))
    cp = _lib.DnCpml()
    for a in range(3):
        cp.b[a] = cp.c[a] = 256
    out = ctypes.c_int32(-1)
    rc = getattr(L, fn)(ctypes.byref(g), fake, fake, 256, ctypes.byref(cp), None, 256, None, 0,
                        4, 4, None, None, ctypes.byref(out))
    assert rc == _lib.DN_EINVAL
    # a record that does not cover the requested steps is rejected too
    rec = _lib.DnCurlRecord(step_stride=8 * 256, t0=2, nslots=2)
    for c in range(3):
        rec.curl[c] = 256
    rc = getattr(L, fn)(ctypes.byref(g), fake, fake, 256, ctypes.byref(cp), ctypes.byref(rec), 256,
                        None, 0, 4, 4, None, None, ctypes.byref(out))
    assert rc == _lib.DN_EINVAL


@pytest.mark.parametrize("name", sorted(_lib.STRUCTS))
def test_ctypes_struct_mirrors_match_the_c_abi(name):
    assert _lib.lib().dn_struct_size(name.encode()) == ctypes.sizeof(_lib.STRUCTS[name])


def test_batch2d_rejects_bad_configs():
    L = _lib.lib()
    cfg = _lib.DnBatch2d(pol=_lib.DN_TM, dtype=_lib.DN_F32, n_inst=1, K=0, tile_rows=16)
    inst = (_lib.DnBatch2dInst * 1)()
    assert L.dn_batch2d_table_bytes(ctypes.byref(cfg), inst) == -1  # K = 0
    cfg.K = 8
    cfg.tile_rows = 12
    assert L.dn_batch2d_table_bytes(ctypes.byref(cfg), inst) == -1  # tile rows
    cfg.tile_rows = 16
    assert L.dn_batch2d_table_bytes(ctypes.byref(cfg), inst) == -1  # empty instance


@pytest.mark.parametrize("bad", [dict(n_ctas=0), dict(missing=-1), dict(spin_limit=0),
                                 dict(spin_limit=(1 << 24) + 1), dict(rounds=0),
                                 dict(bar=None), dict(status=None), dict(bar=8)])
def test_barrier_selftest_rejects_bad_arguments_before_any_launch(bad):
    L = _lib.lib()
    a = dict(n_ctas=4, missing=0, spin_limit=1024, rounds=1, bar=4096, status=8192)
    a.update(bad)
    rc = L.dn_batch2d_barrier_selftest(a["n_ctas"], a["missing"], a["spin_limit"], a["rounds"],
                                       a["bar"], a["status"], None)
    assert rc == _lib.DN_EINVAL


def test_batch2d_requires_16_byte_rows_and_arrays():
    """The batched kernels move rows in 16-byte chunks: an instance whose
    pitch or arrays are not 16-byte aligned is refused before any launch
    (the pointers are only checked, never dereferenced, here)."""
    L = _lib.lib()
    cfg = _lib.DnBatch2d(pol=_lib.DN_TM, dtype=_lib.DN_F32, n_inst=1, K=8, tile_rows=16)

    def inst(pitch=40, ce=0x10000):
        a = (_lib.DnBatch2dInst * 1)()
        i = a[0]
        i.H, i.W, i.pitch, i.n_steps = 20, 37, pitch, 10
        i.src_comp = i.mon_comp = _lib.DN_NONE
        i.dt, i.dl = 1.0, 20.0
        i.ce = ce
        for k in range(2):
            i.b[k], i.c[k] = 0x20000 + 0x100 * k, 0x30000 + 0x100 * k
            for c in range(3):
                i.f[k][c] = 0x40000 + 0x1000 * (3 * k + c)
        return a

    assert L.dn_batch2d_table_bytes(ctypes.byref(cfg), inst()) > 0
    assert L.dn_batch2d_table_bytes(ctypes.byref(cfg), inst(pitch=37)) == -1  # 148-byte rows
    assert L.dn_batch2d_table_bytes(ctypes.byref(cfg), inst(ce=0x10004)) == -1  # misaligned


def test_step_tables_shorter_than_the_run_are_rejected_before_any_launch():
    """The waveform, the monitor phase table and the probe output are indexed
    by the absolute step and carry their length (n_t): a forward run of steps
    t0 .. t0+nsteps-1 past it, or a reverse sweep past a monitor's table, is
    refused on the host (the fake pointers are never dereferenced)."""
    L = _lib.lib()
    out = ctypes.c_int32(-1)
    cp = _lib.DnCpml()
    for a in range(3):
        cp.b[a] = cp.c[a] = 256
    cell = _lib.box((0, 0, 0), (1, 1, 1))
    for fn, D in (("dn_fdtd2d_run", 1), ("dn_fdtd3d_run", 8)):
        g = _grid(D=D, axes=0, pitch_y=32, pitch_z=256)
        fake = _lib.PTR6(*([256] * 6))
        run = getattr(L, fn)
        src = _lib.DnSource(component=_lib.DN_EZ, box=cell, wave=256, n_t=10)
        mon = (_lib.DnMonitor * 1)()
        mon[0] = _lib.DnMonitor(component=_lib.DN_EZ, box=cell, n_freq=1, phase=256, acc=256,
                                n_t=10)
        probe = _lib.DnProbe(component=_lib.DN_EZ, out=256, n_t=10)
        # t0 + nsteps = 11 > 10 for each table in turn
        assert run(ctypes.byref(g), fake, fake, 256, ctypes.byref(cp), ctypes.byref(src), None, 0,
                   None, None, 5, 6, None, None, ctypes.byref(out)) == _lib.DN_EINVAL
        assert run(ctypes.byref(g), fake, fake, 256, ctypes.byref(cp), None, mon, 1, None, None, 5,
                   6, None, None, ctypes.byref(out)) == _lib.DN_EINVAL
        assert run(ctypes.byref(g), fake, fake, 256, ctypes.byref(cp), None, None, 0,
                   ctypes.byref(probe), None, 5, 6, None, None, ctypes.byref(out)) == \
            _lib.DN_EINVAL
        # a disabled source / probe carries no table and is not checked
        off = _lib.DnSource(component=_lib.DN_NONE)
        assert off.n_t == 0
    for fn, D in (("dn_fdtd2d_adjoint", 1), ("dn_fdtd3d_adjoint", 8)):
        g = _grid(D=D, axes=0, pitch_y=32, pitch_z=256)
        fake = _lib.PTR6(*([256] * 6))
        rec = _lib.DnCurlRecord(step_stride=8 * 256, t0=0, nslots=16)
        for c in range(3):
            rec.curl[c] = 256
        mon = (_lib.DnMonitor * 1)()
        mon[0] = _lib.DnMonitor(component=_lib.DN_EZ, box=cell, n_freq=1, phase=256, acc=256,
                                n_t=10)
        # reverse steps 10 and 9: step 10 is beyond the 10-row phase table
        assert getattr(L, fn)(ctypes.byref(g), fake, fake, 256, ctypes.byref(cp),
                              ctypes.byref(rec), 256, mon, 1, 11, 2, None, None,
                              ctypes.byref(out)) == _lib.DN_EINVAL


@pytest.mark.parametrize("bad", ["n0", "n33", "status", "dtype", "pitch", "ptr"])
def test_check_finite_rejects_bad_spans_before_any_launch(bad):
    L = _lib.lib()
    n = 33 if bad == "n33" else 1
    arr = (_lib.DnSpan * 33)()
    for i in range(33):
        arr[i] = _lib.DnSpan(ptr=4096, dtype=_lib.DN_F32, rows=4, cols=8, pitch=8)
    if bad == "dtype":
        arr[0].dtype = 7
    if bad == "pitch":
        arr[0].pitch = 4
    if bad == "ptr":
        arr[0].ptr = None
    rc = L.dn_check_finite(arr, 0 if bad == "n0" else n, None if bad == "status" else 8192, None)
    assert rc == _lib.DN_EINVAL


def test_watchdog_spans_cover_tensors_exactly():
    """Host side of the watchdog: a contiguous tensor becomes 1024-element
    rows plus a remainder row; a narrowed padded field keeps its pitch."""
    import torch

    t = torch.zeros(2500, dtype=torch.float64)
    sp = _lib.spans(t)
    assert [(s.rows, s.cols, s.pitch) for s in sp] == [(2, 1024, 1024), (1, 452, 452)]
    assert sp[1].ptr == t.data_ptr() + 2048 * 8 and sp[0].dtype == _lib.DN_F64
    padded = torch.zeros(2, 5, 7, 32, dtype=torch.float32)
    v = padded[1, :, :, :20]
    (s,) = _lib.spans(v)
    assert (s.rows, s.cols, s.pitch, s.dtype) == (35, 20, 32, _lib.DN_F32)
    assert s.ptr == v.data_ptr()
    with pytest.raises(ValueError):
        _lib.spans(padded[:, 1])  # two set strides that do not fold into rows
    with pytest.raises(ValueError):
        _lib.spans(torch.zeros(4, dtype=torch.int32))


def test_noalloc_refuses_a_pitch_whose_size_would_wrap():
    """H * pitch * 4 bytes would wrap 64 bits to a small number; the
    allocation-free run refuses it as too large before any CUDA call."""
    L = _lib.lib()
    g = _grid(H=4, W=8, pitch_y=(1 << 62) + 8)
    fake = _lib.PTR6(*([256] * 6))
    cp = _lib.DnCpml()
    for a in range(3):
        cp.b[a] = cp.c[a] = 256
    rc = L.dn_fdtd2d_run_noalloc(ctypes.byref(g), fake, 256, ctypes.byref(cp), None, None, 0,
                                 None, 0, 1, None, None)
    assert rc == _lib.DN_ENOMEM
