"""Batched 2-D FDTD: many independent grids in one persistent launch.

The reference solves one grid per ``FDTDSolver2D`` object with a Python step
loop (``diffnano/solvers/fdtd2d.py:309-357``).  Design studies need many small
to medium grids at once -- robust erosion/dilation variants of a design,
wavelength sweeps -- of different sizes and step counts.  ``FDTDBatch2D``
advances all of them in one persistent cooperative kernel
(``dn_batch2d_forward``) and differentiates all of them in a second one
(``dn_batch2d_backward``: checkpoint-segment replay + reverse steps), with the
same step arithmetic as the single-grid kernels.  Each instance is described
by the reference's own constructor arguments and source dict, plus one DFT
line/point/box monitor on its injected field.

``forward`` is differentiable with respect to every instance's eps;
``forward_graphed`` records the eps upload, reset and persistent launch in a
CUDA graph and replays it when the same batch is solved repeatedly (design
iterations).  The tile height is
chosen by ``autotune_tile_rows`` (measured, cached per device and batch
signature).  Gradient-free solves of grids that fit a thread-block cluster's
shared memory run one cluster per grid (``dn_batch2d_forward_cluster``) unless
``cluster=False``; large batches stream faster through the persistent kernel.
Batches of identical grids (same shape, steps, time step, wavelength and
monitor) keep their fields, coefficients and monitor sums in batch-wide
tensors, so eps upload, reset and outputs are one tensor operation each.
"""

from __future__ import annotations

import ctypes
import hashlib
import json
import math
import os
from dataclasses import dataclass, field

import torch

from diffnano_b200 import _lib
from diffnano_b200.solvers import _setup
from diffnano_b200.solvers._engine import compute_device, padded_width

F64 = torch.float64


@dataclass
class BatchInstance:
    """One grid of a batch (the reference's ``FDTDSolver2D`` arguments)."""

    grid_shape: tuple
    n_steps: int
    dl: float = 20.0
    wavelength_nm: float = 1550.0
    pml_layers: int = 10
    courant: float = 0.5
    source: dict = field(default_factory=lambda: {"type": "gaussian_pulse"})
    monitor: dict | None = None  # {"row"|"col"|"pos"|"box": ..., "wavelengths_nm": [...]}

    @property
    def dt(self) -> float:
        return self.courant * self.dl / math.sqrt(2.0)

    @property
    def omega(self) -> float:
        return 2 * math.pi / self.wavelength_nm


class _Inst:
    """Device buffers of one instance."""

    def __init__(self, spec: BatchInstance, pol: int, dtype, dev, K: int, grad: bool,
                 shared: dict | None = None, views: tuple | None = None):
        H, W = spec.grid_shape
        self.spec, self.H, self.W = spec, H, W
        self.Wp = padded_width(W)
        kw = dict(dtype=dtype, device=dev)
        T = spec.n_steps
        # views = (f, ce, acc): slices of batch-wide tensors (uniform batches)
        if views is not None:
            self.f, self.ce = views[0], views[1]
        else:
            self.f = torch.zeros((2, 3, H, self.Wp), **kw)
            self.ce = torch.zeros((H, self.Wp), **kw)
        # read-only tables, shared by instances with the same set-up
        key = json.dumps([H, W, T, spec.pml_layers, spec.dl, spec.dt, spec.omega, str(dtype),
                          spec.source, spec.monitor], sort_keys=True, default=str)
        shared = {} if shared is None else shared
        if key not in shared:
            prof = [tuple(t.to(dev) for t in _setup.cpml_profile(n, spec.pml_layers, spec.dl,
                                                                 spec.dt)) for n in (H, W)]
            wave = _setup.waveform_table(T, spec.dt, spec.omega, spec.source).to(**kw)
            phase = None
            if spec.monitor is not None:
                wl = [float(w) for w in spec.monitor.get("wavelengths_nm", [spec.wavelength_nm])]
                phase = _setup.dft_phase_table(T, spec.dt, wl).to(dev)
            shared[key] = (prof, wave, phase)
        self.prof, self.wave, phase = shared[key]
        self.src_box = _setup.source_box_2d((H, W), spec.source)
        self.mon_box, self.phase, self.acc, self.nf = None, None, None, 0
        if spec.monitor is not None:
            box = _setup.monitor_box(spec.monitor, (1, H, W), False)
            wl = [float(w) for w in spec.monitor.get("wavelengths_nm", [spec.wavelength_nm])]
            self.mon_box, self.nf = box, len(wl)
            self.mon_shape = tuple(b - a for a, b in box[1:])
            cells = self.mon_shape[0] * self.mon_shape[1]
            self.phase = phase
            self.acc = views[2] if views is not None else \
                torch.zeros((self.nf, cells, 2), dtype=F64, device=dev)
        self.grad_enabled = grad
        nck = max(0, math.ceil(T / K) - 1)
        self.ckpt = torch.zeros((max(1, nck), 3, H, self.Wp), **kw) if grad else None
        ncurl = 1 if pol == _lib.DN_TM else 2
        self.curl = torch.zeros((min(K, T), ncurl, H, self.Wp), **kw) if grad else None
        self.lam = torch.zeros((2, 3, H, self.Wp), **kw) if grad else None
        self.grad = torch.zeros((H, self.Wp), dtype=F64, device=dev) if grad else None
        self.gmon = None

    def struct(self, pol: int) -> _lib.DnBatch2dInst:
        s = _lib.DnBatch2dInst()
        sp = self.spec
        s.H, s.W, s.pitch, s.n_steps = self.H, self.W, self.Wp, sp.n_steps
        first = _lib.DN_EZ if pol == _lib.DN_TM else _lib.DN_HZ
        s.src_comp = first if self.src_box is not None else _lib.DN_NONE
        if self.src_box is not None:
            s.src_box = _lib.box([a for a, _ in self.src_box], [b for _, b in self.src_box])
        s.wave = self.wave.data_ptr()
        for k in range(2):
            for c in range(3):
                s.f[k][c] = self.f[k, c].data_ptr()
                if self.lam is not None:
                    s.lam[k][c] = self.lam[k, c].data_ptr()
        s.ce = self.ce.data_ptr()
        s.b[0], s.c[0] = self.prof[0][0].data_ptr(), self.prof[0][1].data_ptr()
        s.b[1], s.c[1] = self.prof[1][0].data_ptr(), self.prof[1][1].data_ptr()
        s.dt, s.dl = sp.dt, sp.dl
        s.mon_comp = _lib.DN_NONE
        if self.mon_box is not None:
            s.mon_comp = first
            s.mon_box = _lib.box([a for a, _ in self.mon_box], [b for _, b in self.mon_box])
            s.n_freq, s.phase, s.acc = self.nf, self.phase.data_ptr(), self.acc.data_ptr()
        if self.grad_enabled:
            s.ckpt, s.curl, s.grad = self.ckpt.data_ptr(), self.curl.data_ptr(), self.grad.data_ptr()
        s.gmon = self.gmon.data_ptr() if self.gmon is not None else None
        return s


def _signature(specs, pol, dtype) -> str:
    key = json.dumps([pol, str(dtype)] + [[*s.grid_shape, s.n_steps] for s in specs])
    return hashlib.sha1(key.encode()).hexdigest()[:16]


def _cache_path() -> str:
    base = os.environ.get("XDG_CACHE_HOME", os.path.join(os.path.expanduser("~"), ".cache"))
    return os.path.join(base, "diffnano_b200", "autotune.json")


class FDTDBatch2D:
    """Many 2-D grids (same polarisation) solved by one persistent launch.

    Parameters
    ----------
    instances : list of BatchInstance
    polarization : "TM" or "TE"
    dtype : torch.float32 (default) or torch.float64
    device : CUDA device to run on
    checkpoint_interval : steps between stored states for the adjoint
        (default sqrt of the longest step count)
    tile_rows : 8, 16 or 32; None lets ``autotune_tile_rows`` choose
    cluster : gradient-free solves with each grid in one 16-CTA thread-block
        cluster: None = when every grid fits, False = never, True = always
        (error if a grid does not fit)
    """

    def __init__(self, instances, polarization: str = "TM", dtype=torch.float32,
                 device="cuda", checkpoint_interval: int | None = None, tile_rows: int | None = None,
                 cluster: bool | None = None):
        if not instances:
            raise ValueError("empty batch")
        self.specs = list(instances)
        self.pol = _lib.DN_TM if polarization.upper() == "TM" else _lib.DN_TE
        if polarization.upper() not in ("TM", "TE"):
            raise ValueError(f"polarization must be 'TM' or 'TE', got {polarization!r}")
        if dtype not in (torch.float32, torch.float64):
            raise ValueError("dtype must be torch.float32 or torch.float64")
        self.dtype = dtype
        self.device = compute_device(device)
        T = max(s.n_steps for s in self.specs)
        self.K = int(checkpoint_interval or max(1, math.ceil(math.sqrt(T))))
        self.tile_rows = tile_rows
        self._insts = None
        self._stack = None
        self._grad_alloc = None
        self._graph = None
        self._ggraph = None
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        # gradient-free solves: whole grids in thread-block clusters when they fit
        # (None = when possible, False = never)
        self.cluster = cluster
        self._cluster = (0, 0)

    # ------------------------------------------------------------------
    def _cfg(self, rows: int, n_inst: int, max_ctas: int) -> _lib.DnBatch2d:
        return _lib.DnBatch2d(pol=self.pol, dtype=_lib.DN_F32 if self.dtype == torch.float32
                              else _lib.DN_F64, n_inst=n_inst, K=self.K, tile_rows=rows,
                              max_ctas=max_ctas)

    def _build(self, grad: bool):
        if self._insts is not None and self._grad_alloc == grad:
            return
        shared: dict = {}
        views = self._stacked_views()
        self._insts = [_Inst(s, self.pol, self.dtype, self.device, self.K, grad, shared,
                             None if views is None else views[n])
                       for n, s in enumerate(self.specs)]
        self._grad_alloc = grad
        self._graph = None
        if self.tile_rows is None:
            self.tile_rows = autotune_tile_rows(self)
        self._pack()

    def _stacked_views(self):
        """Uniform batches (every instance with the same grid, step count, time
        step, wavelength and monitor) keep fields, coefficients and monitor
        sums in three batch-wide tensors, so that eps upload, reset and outputs
        are one tensor operation each instead of one per instance; returns the
        per-instance views, or None."""
        self._stack = None
        s0 = self.specs[0]

        def key(sp):
            return json.dumps([list(sp.grid_shape), sp.n_steps, sp.dt, sp.wavelength_nm,
                               sp.monitor], sort_keys=True, default=str)

        k0 = key(s0)
        if len(self.specs) < 2 or any(key(sp) != k0 for sp in self.specs[1:]):
            return None
        n = len(self.specs)
        H, W = s0.grid_shape
        Wp = padded_width(W)
        kw = dict(dtype=self.dtype, device=self.device)
        f = torch.zeros((n, 2, 3, H, Wp), **kw)
        ce = torch.zeros((n, H, Wp), **kw)
        acc = None
        if s0.monitor is not None:
            box = _setup.monitor_box(s0.monitor, (1, H, W), False)
            nf = len(s0.monitor.get("wavelengths_nm", [s0.wavelength_nm]))
            cells = (box[1][1] - box[1][0]) * (box[2][1] - box[2][0])
            acc = torch.zeros((n, nf, cells, 2), dtype=F64, device=self.device)
        self._stack = (f, ce, acc)
        return [(f[b], ce[b], None if acc is None else acc[b]) for b in range(n)]

    def _pack(self):
        # recorded graphs launch with the device table they were captured
        # with: a new table (new pointers) makes them stale
        self._graph = None
        self._ggraph = None
        L = _lib.lib()
        arr = (_lib.DnBatch2dInst * len(self._insts))(*[i.struct(self.pol) for i in self._insts])
        cols = 128 if self.dtype == torch.float32 else 64  # tile width: 32 lanes x 16 bytes
        tiles = sum(((i.W + cols - 1) // cols) * ((i.H + self.tile_rows - 1) // self.tile_rows)
                    for i in self._insts)
        self.cfg = self._cfg(self.tile_rows, len(self._insts), tiles)
        smem = ctypes.c_int64(0)
        cl = int(L.dn_batch2d_cluster_size(ctypes.byref(self.cfg), arr, ctypes.byref(smem)))
        self._cluster = (cl, int(smem.value)) if cl > 0 else (0, 0)
        if self.cluster and not self._cluster[0]:
            raise ValueError("an instance is too large for a thread-block cluster")
        nbytes = int(L.dn_batch2d_table_bytes(ctypes.byref(self.cfg), arr))
        if nbytes < 0:
            raise ValueError("invalid batch description")
        host = (ctypes.c_ubyte * nbytes)()
        _lib.check("dn_batch2d_pack", L.dn_batch2d_pack(ctypes.byref(self.cfg), arr, host, nbytes))
        self.table = torch.frombuffer(bytearray(host), dtype=torch.uint8).to(self.device)

    def uses_cluster(self, grad: bool) -> bool:
        """Whether a forward with / without gradient runs the cluster kernel."""
        return (not grad) and self.cluster is not False and self._cluster[0] > 0

    def _launch(self, fwd: bool, grad: bool = True):
        L = _lib.lib()
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            if fwd and self.uses_cluster(grad):
                fn = "dn_batch2d_forward_cluster"
                rc = L.dn_batch2d_forward_cluster(ctypes.byref(self.cfg), self.table.data_ptr(),
                                                  self._cluster[0], self._cluster[1],
                                                  ctypes.c_void_p(stream))
            else:
                fn = "dn_batch2d_forward" if fwd else "dn_batch2d_backward"
                rc = getattr(L, fn)(ctypes.byref(self.cfg), self.table.data_ptr(),
                                    self.status.data_ptr(), ctypes.c_void_p(stream))
        _lib.check(fn, rc)

    def _reset(self):
        if self._stack is not None:
            self._stack[0].zero_()
            if self._stack[2] is not None:
                self._stack[2].zero_()
            return
        for i in self._insts:
            i.f.zero_()
            if i.acc is not None:
                i.acc.zero_()

    def _set_eps(self, eps_list):
        if self._stack is not None:
            i0, n = self._insts[0], len(self._insts)
            eps = eps_list if isinstance(eps_list, torch.Tensor) else \
                torch.stack([e.detach().to(self.device, F64) for e in eps_list])
            if eps.shape[0] != n or tuple(eps.shape[-2:]) != (i0.H, i0.W):
                raise ValueError(f"eps shape {tuple(eps.shape)} != {n} grids {(i0.H, i0.W)}")
            eps = eps.detach().to(self.device, F64).reshape(n, i0.H, i0.W)
            self._stack[1][:, :, : i0.W] = (i0.spec.dt / eps).to(self.dtype)
            return
        for i, e in zip(self._insts, eps_list):
            if tuple(e.shape[-2:]) != (i.H, i.W):
                raise ValueError(f"eps shape {tuple(e.shape)} != grid {(i.H, i.W)}")
            i.ce[:, : i.W] = (i.spec.dt / e.detach().to(self.device, F64).reshape(i.H, i.W)).to(self.dtype)

    def run_forward(self, eps_list, grad: bool = False):
        """All steps of all instances (no autograd); returns (fields, dfts)."""
        self._build(grad)
        self._set_eps(eps_list)
        self._reset()
        self._launch(True, grad)
        return self._outputs()

    def _outputs(self):
        if self._stack is not None:
            i0, n = self._insts[0], len(self._insts)
            fields = list(self._stack[0][:, i0.spec.n_steps % 2, 0, :, : i0.W].clone().unbind(0))
            dfts = [None] * n
            if self._stack[2] is not None:
                d = torch.view_as_complex(self._stack[2]).reshape(n, i0.nf, *i0.mon_shape)
                dfts = list(d.clone().unbind(0))
            return fields, dfts
        fields, dfts = [], []
        for i in self._insts:
            fields.append(i.f[i.spec.n_steps % 2, 0, :, : i.W].clone())
            if i.acc is not None:
                dfts.append(torch.view_as_complex(i.acc).reshape(i.nf, *i.mon_shape).clone())
            else:
                dfts.append(None)
        return fields, dfts

    def run_backward(self, g_fields, g_dfts):
        """Reverse sweep; returns dL/d(dt/eps) per instance (FP64)."""
        for i, gf, gd in zip(self._insts, g_fields, g_dfts):
            i.lam.zero_()
            i.grad.zero_()
            if gf is not None:
                i.lam[i.spec.n_steps % 2, 0, :, : i.W] = gf.to(self.device, self.dtype)
            i.gmon = None
            if gd is not None and i.acc is not None:
                i.gmon = torch.view_as_real(gd.to(self.device, torch.complex128)).reshape(
                    i.nf, -1, 2).contiguous()
        self._pack()  # gradient pointers may have changed
        self._launch(False)
        return [i.grad[:, : i.W] for i in self._insts]

    def forward_graphed(self, eps_list):
        """``run_forward`` through a CUDA graph: the first call records the
        eps upload, state reset and persistent launch; later calls copy the
        new eps into the recorded input buffers and replay.  No autograd."""
        self._build(False)
        if self._graph is None:
            self._static_eps = [e.detach().to(self.device, F64).clone() for e in eps_list]
            side = torch.cuda.Stream(self.device)
            side.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(side):
                self._graph_body()  # warm-up outside the capture
            torch.cuda.current_stream(self.device).wait_stream(side)
            torch.cuda.synchronize(self.device)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._graph_body()
            self._graph = g
        for dst, e in zip(self._static_eps, eps_list):
            dst.copy_(e.detach())
        self._graph.replay()
        self.check_status()
        return self._outputs()

    def fom_gradient_graphed(self, eps_list):
        """FOM = sum |DFT|^2 of every instance's monitor and dFOM/deps, as one
        CUDA-graph replay: the first call records eps upload, state reset,
        the persistent forward launch (checkpoints on), the seeding of the
        adjoint with dFOM/dDFT = 2 DFT, the persistent backward launch and
        dFOM/deps = -(dt/eps^2) dFOM/d(dt/eps); later calls copy the new eps
        into the recorded input buffers and replay.  Returns (per-instance
        FOM tensor (FP64), list of dFOM/deps (FP64, one per instance)); the
        results are views of graph-owned buffers, overwritten by the next
        call.  No autograd."""
        self._build(True)
        if any(i.acc is None for i in self._insts):
            raise ValueError("fom_gradient_graphed needs a monitor on every instance")
        if getattr(self, "_ggraph", None) is None:
            self._g_eps = [e.detach().to(self.device, F64).clone() for e in eps_list]
            for i in self._insts:
                i.gmon = torch.zeros_like(i.acc)
            self._pack()
            self._g_fom = torch.zeros(len(self._insts), dtype=F64, device=self.device)
            self._g_out = [torch.zeros(i.H, i.W, dtype=F64, device=self.device)
                           for i in self._insts]
            side = torch.cuda.Stream(self.device)
            side.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(side):
                self._grad_body()  # warm-up outside the capture
            torch.cuda.current_stream(self.device).wait_stream(side)
            torch.cuda.synchronize(self.device)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._grad_body()
            self._ggraph = g
        for dst, e in zip(self._g_eps, eps_list):
            dst.copy_(e.detach())
        self._ggraph.replay()
        self.check_status(grads=True)
        return self._g_fom, self._g_out

    def _grad_body(self):
        for i, e in zip(self._insts, self._g_eps):
            i.ce[:, : i.W] = (i.spec.dt / e).to(self.dtype)
        self._reset()
        self._launch(True, True)
        for n, i in enumerate(self._insts):
            self._g_fom[n] = (i.acc * i.acc).sum()
            torch.mul(i.acc, 2.0, out=i.gmon)
            i.lam.zero_()
            i.grad.zero_()
        self._launch(False)
        for i, e, out in zip(self._insts, self._g_eps, self._g_out):
            torch.mul(i.grad[:, : i.W], -(i.spec.dt) / (e * e), out=out)

    def _graph_body(self):
        for i, e in zip(self._insts, self._static_eps):
            i.ce[:, : i.W] = (i.spec.dt / e).to(self.dtype)
        self._reset()
        self._launch(True, False)

    def check_status(self, grads: bool = False):
        """Scan the final fields and monitor sums (the gradients after a
        backward sweep) for NaN/Inf with the watchdog kernel, then raise if
        a kernel or the scan recorded an error (synchronises)."""
        if self._insts is not None:
            if grads:
                ts = [i.grad[:, : i.W] for i in self._insts if i.grad is not None]
            else:
                ts = [i.f[i.spec.n_steps % 2, :, :, : i.W] for i in self._insts]
                if self._stack is not None:  # batch-wide monitor sums: one tensor
                    ts.append(self._stack[2])
                else:
                    ts += [i.acc for i in self._insts if i.acc is not None]
            with torch.cuda.device(self.device):
                _lib.check_finite(ts, self.status,
                                  torch.cuda.current_stream(self.device).cuda_stream)
        s = int(self.status.item())
        if s != _lib.DN_OK:
            self.status.zero_()
            _lib.check("batched FDTD", s)

    # ------------------------------------------------------------------
    def forward(self, eps_list):
        """Differentiable solve of every instance.

        Returns ``(fields, dfts)``: per instance the final injected-field
        component ``(H, W)`` (Ez for TM, Hz for TE) and the complex monitor
        DFT ``(L, rows, cols)`` (None without a monitor).
        """
        eps_list = list(eps_list)
        if len(eps_list) != len(self.specs):
            raise ValueError("one eps per instance")
        needs = torch.is_grad_enabled() and any(e.requires_grad for e in eps_list)
        if not needs:
            with torch.no_grad():
                out = self.run_forward(eps_list, grad=False)
            self.check_status()
            return out
        outs = _BatchFDTD.apply(self, len(eps_list), *eps_list)
        n = len(eps_list)
        fields = list(outs[:n])
        dfts = []
        for i, d in zip(self._insts, outs[n:]):
            dfts.append(torch.view_as_complex(d.reshape(-1, 2)).reshape(i.nf, *i.mon_shape)
                        if i.acc is not None else None)
        return fields, dfts


class _BatchFDTD(torch.autograd.Function):
    @staticmethod
    def forward(ctx, batch, n, *eps_list):
        fields, dfts = batch.run_forward(eps_list, grad=True)
        batch.check_status()
        ctx.batch, ctx.n = batch, n
        ctx.save_for_backward(*eps_list)
        flat = [torch.view_as_real(d).reshape(-1) if d is not None
                else torch.zeros(0, dtype=F64, device=batch.device) for d in dfts]
        return (*fields, *flat)

    @staticmethod
    def backward(ctx, *grads):
        batch, n = ctx.batch, ctx.n
        eps_list = ctx.saved_tensors
        g_fields = list(grads[:n])
        g_dfts = []
        for i, g in zip(batch._insts, grads[n:]):
            g_dfts.append(torch.view_as_complex(g.reshape(-1, 2).contiguous())
                          if (g is not None and i.acc is not None) else None)
        gce = batch.run_backward(g_fields, g_dfts)
        batch.check_status(grads=True)
        out = []
        for e, gc, i in zip(eps_list, gce, batch._insts):
            ed = e.detach().to(gc.device, F64).reshape(gc.shape)
            out.append((-(i.spec.dt / (ed * ed)) * gc).reshape(e.shape).to(e.device, e.dtype))
        return (None, None, *out)


def autotune_tile_rows(batch: FDTDBatch2D, candidates=(8, 16, 32), probe_steps: int = 64) -> int:
    """Pick the tile height for a batch by timing a short forward of each
    candidate on this device; results are cached per (device, batch
    signature) in ``~/.cache/diffnano_b200/autotune.json``."""
    dev_name = torch.cuda.get_device_name(batch.device)
    key = f"{dev_name}|batch2d|{_signature(batch.specs, batch.pol, batch.dtype)}"
    path = _cache_path()
    try:
        with open(path) as fh:
            cache = json.load(fh)
    except (OSError, ValueError):
        cache = {}
    if key in cache and int(cache[key]["tile_rows"]) in candidates:
        return int(cache[key]["tile_rows"])
    probe = [BatchInstance(**{**s.__dict__, "n_steps": min(s.n_steps, probe_steps),
                              "monitor": None}) for s in batch.specs]
    times = {}
    for rows in candidates:
        b = FDTDBatch2D(probe, "TM" if batch.pol == _lib.DN_TM else "TE", batch.dtype,
                        batch.device, tile_rows=rows)
        eps = [torch.full(s.grid_shape, 2.0, dtype=F64) for s in probe]
        b.run_forward(eps)  # warm-up
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b._launch(True)
        e1.record()
        torch.cuda.synchronize(batch.device)
        b.check_status()
        times[rows] = e0.elapsed_time(e1)
    best = min(times, key=times.get)
    cache[key] = {"tile_rows": best, "ms": {str(k): v for k, v in times.items()}}
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as fh:
            json.dump(cache, fh, indent=1)
    except OSError:
        pass
    return best
