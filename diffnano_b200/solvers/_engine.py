"""Device state and kernel driver shared by the 2-D and 3-D solvers.

An :class:`Engine` owns, on one CUDA device, everything the C ABI needs for
one solver configuration: two ping-pong field sets ``(6, D, H, Wp)`` (rows
padded to ``Wp``, a multiple of 32 elements, so every row starts 128-byte
aligned and TMA boxes are legal), the per-cell coefficient ``dt/eps``, the
CPML profiles, the source waveform table, DFT-monitor phase tables and FP64
accumulators, and a probe buffer.  It runs steps through
``dn_fdtd2d_run`` / ``dn_fdtd3d_run`` on the current torch stream.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import torch

from diffnano_b200 import _lib
from diffnano_b200.solvers import _setup

F64 = torch.float64


def to_result_device(t: torch.Tensor, device) -> torch.Tensor:
    """``t`` (on the compute GPU) moved to a solver's result ``device``.

    A CPU result goes into page-locked memory taken from torch's caching host
    allocator (the blocks of results the caller has dropped are reused), with
    an asynchronous copy and a sync of the copying stream: a 201 MB field
    comes back in ~4 ms instead of ~90 ms through a pageable staging copy.
    The copy stays differentiable (``copy_`` records its backward)."""
    dev = torch.device(device)
    if dev.type != "cpu" or not t.is_cuda:
        return t.to(dev)
    out = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    with torch.cuda.device(t.device):
        out.copy_(t, non_blocking=True)
        torch.cuda.current_stream(t.device).synchronize()
    return out


def compute_device(device) -> torch.device:
    """CUDA device the kernels run on for a solver built with ``device``.

    The reference runs wherever ``device`` says, CPU included.  These
    kernels exist only for CUDA (sm_100a): a CUDA ``device`` is used as is;
    any other ``device`` names where inputs and results live, and the
    computation runs on the current CUDA device.  There is no CPU path.
    """
    dev = torch.device(device)
    if not torch.cuda.is_available():
        raise RuntimeError(
            "diffnano_b200 runs its FDTD kernels on a CUDA GPU (sm_100a) and has no CPU path; "
            "no CUDA device is visible")
    if dev.type == "cuda":
        return dev if dev.index is not None else torch.device("cuda", torch.cuda.current_device())
    return torch.device("cuda", torch.cuda.current_device())


def padded_width(W: int) -> int:
    return (W + 31) // 32 * 32


@dataclass
class MonitorSpec:
    name: str
    component: int
    box: tuple  # ((z0,z1),(y0,y1),(x0,x1))
    wavelengths: list
    cells: int = field(init=False)

    def __post_init__(self):
        self.cells = 1
        for a, b in self.box:
            self.cells *= b - a

    @property
    def shape(self):
        return tuple(b - a for a, b in self.box)


class Engine:
    """Device state + launcher for one grid / source / monitor configuration."""

    def __init__(self, *, is3d: bool, shape, dl: float, dt: float, pml_layers: int,
                 dtype: torch.dtype, device: torch.device, n_steps: int, wave: torch.Tensor,
                 src_box, src_comp: int, monitors=(), probe=None, pol: int = _lib.DN_TM,
                 axes: int = _lib.DN_AXES_REFERENCE):
        if dtype not in (torch.float32, torch.float64):
            raise ValueError(f"dtype must be torch.float32 or torch.float64, got {dtype}")
        self.is3d = is3d
        self.shape3 = tuple(int(v) for v in (shape if is3d else (1, *shape)))
        D, H, W = self.shape3
        self.Wp = padded_width(W)
        self.dtype, self.device = dtype, device
        self.dl, self.dt, self.n_steps = float(dl), float(dt), int(n_steps)
        self.pol, self.axes = pol, axes
        kw = dict(dtype=dtype, device=device)
        self.A = torch.zeros((6, D, H, self.Wp), **kw)
        self.B = torch.zeros((6, D, H, self.Wp), **kw)
        self.ce = torch.zeros((D, H, self.Wp), **kw)
        self.cur_b = False

        # CPML profiles: axis 0 = z (D), 1 = y (H), 2 = x (W)
        self.prof = []
        for a, n in enumerate(self.shape3):
            if a == 0 and not is3d:
                self.prof.append(None)
                continue
            b, c = _setup.cpml_profile(n, pml_layers, dl, dt)
            self.prof.append((b.to(device), c.to(device)))
        self.cpml = _lib.DnCpml()
        for a in range(3):
            if self.prof[a] is not None:
                self.cpml.b[a] = self.prof[a][0].data_ptr()
                self.cpml.c[a] = self.prof[a][1].data_ptr()

        self.grid = _lib.DnGrid(D=D, H=H, W=W, dtype=_lib.DN_F32 if dtype == torch.float32 else _lib.DN_F64,
                                pitch_y=self.Wp, pitch_z=H * self.Wp, dt=self.dt, dl=self.dl,
                                axes=axes, pol=pol)

        # source
        self.wave = wave.to(device=device, dtype=dtype).contiguous()
        self.src = _lib.DnSource(component=_lib.DN_NONE)
        if src_box is not None and src_comp != _lib.DN_NONE:
            self.src.component = src_comp
            self.src.box = _lib.box([a for a, _ in src_box], [b for _, b in src_box])
            self.src.wave = self.wave.data_ptr()
            self.src.n_t = self.wave.numel()

        # monitors
        if len(monitors) > _lib.DN_MAX_MONITORS:
            raise ValueError(f"at most {_lib.DN_MAX_MONITORS} monitors per solve")
        self.monitors = list(monitors)
        self.phases, self.accs = [], []
        self.mon_arr = (_lib.DnMonitor * max(1, len(self.monitors)))()
        for m, spec in enumerate(self.monitors):
            if not 1 <= len(spec.wavelengths) <= _lib.DN_MAX_FREQS:
                raise ValueError(f"a monitor takes 1..{_lib.DN_MAX_FREQS} wavelengths")
            ph = _setup.dft_phase_table(self.n_steps, self.dt, spec.wavelengths).to(device)
            acc = torch.zeros((len(spec.wavelengths), spec.cells, 2), dtype=F64, device=device)
            self.phases.append(ph)
            self.accs.append(acc)
            M = self.mon_arr[m]
            M.component = spec.component
            M.box = _lib.box([a for a, _ in spec.box], [b for _, b in spec.box])
            M.n_freq = len(spec.wavelengths)
            M.phase = ph.data_ptr()
            M.acc = acc.data_ptr()
            M.n_t = ph.shape[0]

        # probe
        self.probe = _lib.DnProbe(component=_lib.DN_NONE)
        self.probe_out = None
        if probe is not None:
            comp, pos = probe
            self.probe_out = torch.zeros(self.n_steps, **kw)
            self.probe.component = comp
            for a in range(3):
                self.probe.pos[a] = int(pos[a])
            self.probe.out = self.probe_out.data_ptr()
            self.probe.n_t = self.probe_out.numel()

        self.status = torch.zeros(1, dtype=torch.int32, device=device)

    # ------------------------------------------------------------------
    def set_eps(self, eps: torch.Tensor) -> None:
        """Per-cell coefficient dt/eps (computed in FP64, stored in the dtype)."""
        e = eps.to(device=self.device).reshape(self.shape3)
        self.ce[..., : self.shape3[2]] = (self.dt / e.to(F64)).to(self.dtype)

    def current(self) -> torch.Tensor:
        return self.B if self.cur_b else self.A

    def field(self, comp: int) -> torch.Tensor:
        """View ``(D, H, W)`` of a component of the current state."""
        return self.current()[comp, :, :, : self.shape3[2]]

    def reset(self) -> None:
        self.A.zero_()
        self.B.zero_()
        self.cur_b = False
        for a in self.accs:
            a.zero_()
        if self.probe_out is not None:
            self.probe_out.zero_()
        self.status.zero_()

    def load_state(self, state: torch.Tensor) -> None:
        self.current().copy_(state)

    @staticmethod
    def _ptrs(t: torch.Tensor):
        return _lib.PTR6(*[t[c].data_ptr() for c in range(6)])

    def run(self, t0: int, nsteps: int, record=None, outputs: bool = True) -> None:
        """Advance ``nsteps`` steps starting at absolute step ``t0``.

        ``record`` (a ``DnCurlRecord``) stores each step's curl terms for the
        adjoint; ``outputs=False`` skips the monitors and the probe (used when
        a segment is replayed for the adjoint, whose DFTs are already known).
        """
        if nsteps <= 0:
            return
        if t0 + nsteps > self.n_steps:
            raise ValueError("step range beyond the precomputed source/monitor tables")
        L = _lib.lib()
        fa, fb = (self.B, self.A) if self.cur_b else (self.A, self.B)
        out = ctypes.c_int32(0)
        fn_name = "dn_fdtd3d_run" if self.is3d else "dn_fdtd2d_run"
        no_probe = _lib.DnProbe(component=_lib.DN_NONE)
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            rc = getattr(L, fn_name)(
                ctypes.byref(self.grid), self._ptrs(fa), self._ptrs(fb), self.ce.data_ptr(),
                ctypes.byref(self.cpml), ctypes.byref(self.src), self.mon_arr,
                len(self.monitors) if outputs else 0,
                ctypes.byref(self.probe if outputs else no_probe),
                ctypes.byref(record) if record is not None else None, int(t0), int(nsteps),
                self.status.data_ptr(), ctypes.c_void_p(stream), ctypes.byref(out))
        _lib.check(fn_name, rc)
        if out.value:
            self.cur_b = not self.cur_b

    # ------------------------------------------------------------------
    # adjoint support
    # ------------------------------------------------------------------
    def eps_components(self):
        """Components whose update carries dt/eps (and so a curl record)."""
        if self.is3d:
            return (_lib.DN_EX, _lib.DN_EY, _lib.DN_EZ)
        return (_lib.DN_EZ,) if self.pol == _lib.DN_TM else (_lib.DN_EX, _lib.DN_EY)

    def curl_buffer(self, nslots: int) -> torch.Tensor:
        """``(3, nslots, D, H, Wp)`` curl storage (only the slots of the
        components that carry eps are written)."""
        D, H, _ = self.shape3
        ncomp = 3 if self.is3d else len(self.eps_components())
        return torch.empty((ncomp, nslots, D, H, self.Wp), dtype=self.dtype, device=self.device)

    def curl_record(self, buf: torch.Tensor, t0: int, nslots: int):
        rec = _lib.DnCurlRecord(step_stride=buf.shape[2] * buf.shape[3] * buf.shape[4], t0=int(t0),
                                nslots=int(nslots))
        comps = self.eps_components()
        for n, c in enumerate(comps):
            slot = c if self.is3d else (2 if c == _lib.DN_EZ else c)
            rec.curl[slot] = buf[n].data_ptr()
        return rec

    def adjoint(self, la: torch.Tensor, lb: torch.Tensor, rec, grad_ce: torch.Tensor, mon_arr,
                n_mon: int, t_end: int, nsteps: int) -> bool:
        """Reverse steps t_end-1 .. t_end-nsteps on adjoint sets la/lb (la
        holds the current adjoint).  Returns True when the result ends in lb."""
        L = _lib.lib()
        out = ctypes.c_int32(0)
        fn_name = "dn_fdtd3d_adjoint" if self.is3d else "dn_fdtd2d_adjoint"
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            rc = getattr(L, fn_name)(
                ctypes.byref(self.grid), self._ptrs(la), self._ptrs(lb), self.ce.data_ptr(),
                ctypes.byref(self.cpml), ctypes.byref(rec), grad_ce.data_ptr(), mon_arr,
                int(n_mon), int(t_end), int(nsteps), self.status.data_ptr(),
                ctypes.c_void_p(stream), ctypes.byref(out))
        _lib.check(fn_name, rc)
        return bool(out.value)

    def check_status(self, extra=()) -> None:
        """Scan the current state of the solver's components, the monitor
        DFTs, the probe series and the ``extra`` tensors for NaN/Inf with the
        watchdog kernel, then raise if a kernel or the scan recorded a
        device-side error (synchronises)."""
        used = ((_lib.DN_EX, _lib.DN_EY, _lib.DN_EZ, _lib.DN_HX, _lib.DN_HY, _lib.DN_HZ)
                if self.is3d else (_lib.DN_EZ, _lib.DN_HX, _lib.DN_HY) if self.pol == _lib.DN_TM
                else (_lib.DN_HZ, _lib.DN_EX, _lib.DN_EY))
        ts = [self.field(c) for c in used] + list(self.accs) + [self.probe_out, *extra]
        with torch.cuda.device(self.device):
            _lib.check_finite(ts, self.status, torch.cuda.current_stream(self.device).cuda_stream)
        s = int(self.status.item())
        if s != _lib.DN_OK:
            _lib.check("device status", s)

    def monitor_dft(self, m: int) -> torch.Tensor:
        """Complex ``(L, *box_shape)`` DFT of monitor ``m`` (complex128); 2-D
        boxes drop their z extent, so a 2-D shape is ``(L, rows, cols)``."""
        spec = self.monitors[m]
        shape = spec.shape if self.is3d else spec.shape[1:]
        return torch.view_as_complex(self.accs[m]).reshape(len(spec.wavelengths), *shape)
