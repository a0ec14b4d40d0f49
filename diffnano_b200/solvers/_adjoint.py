"""Forward driver and the autograd bridge to the hand-written adjoint kernels.

The reference differentiates its FDTD with PyTorch autograd through every
time step (``diffnano/solvers/fdtd2d.py:309-410``, ``fdtd3d.py:471-562``),
or, with ``backward="time_reversal"``, by re-running the forward under
autograd inside a custom ``autograd.Function`` (``fdtd3d.py:88-219``).  Here
both modes are one ``torch.autograd.Function`` whose backward is the discrete
adjoint of the kernels' own step:

* forward: all T steps run in the CUDA kernels; when a gradient is needed the
  state is copied every K steps (K = sqrt(T), or T / checkpoint_segments with
  ``use_checkpoint``);
* backward: for each segment, last first, the segment is replayed from its
  checkpoint with the curl term of every step recorded, then the adjoint
  kernel runs the segment's steps backwards, accumulating dL/d(dt/eps) in
  FP64; dL/deps = -(dt/eps^2) dL/d(dt/eps).

Peak memory is the checkpoints (T/K states) plus one segment of curl records
(K x 3 fields), not the T-step autograd graph.
"""

from __future__ import annotations

import torch

from diffnano_b200 import _lib
from diffnano_b200.solvers._common import checkpoint_interval

F64 = torch.float64


def _outputs(eng, out_names):
    comps = [_lib.COMPONENTS[n] for n in out_names]
    f = torch.stack([eng.field(c) if eng.is3d else eng.field(c)[0] for c in comps])
    dfts = [eng.monitor_dft(m).clone() for m in range(len(eng.monitors))]
    return f, dfts


class _Runner:
    """Forward with checkpoints and the adjoint sweep for one Engine."""

    def __init__(self, eng, out_names, interval: int):
        self.eng = eng
        self.out_names = tuple(out_names)
        self.K = max(1, int(interval))
        self.checkpoints = {}

    def forward(self, eps_dev: torch.Tensor, save: bool):
        eng = self.eng
        eng.reset()
        eng.set_eps(eps_dev)
        T, K = eng.n_steps, self.K
        t = 0
        while t < T:
            n = min(K, T - t)
            if save and t > 0:
                self.checkpoints[t] = eng.current().clone()
            eng.run(t, n)
            t += n
        f, dfts = _outputs(eng, self.out_names)
        eng.check_status()
        mon = torch.cat([torch.view_as_real(d).reshape(-1) for d in dfts]) if dfts else \
            torch.zeros(0, dtype=F64, device=eng.device)
        return f, mon

    def adjoint(self, g_field, g_mon) -> torch.Tensor:
        """dL/d(dt/eps) as an FP64 ``(D, H, W)`` tensor."""
        eng = self.eng
        D, H, W = eng.shape3
        kw = dict(dtype=eng.dtype, device=eng.device)
        la = torch.zeros((6, D, H, eng.Wp), **kw)
        lb = torch.zeros((6, D, H, eng.Wp), **kw)
        if g_field is not None:
            g = g_field.to(device=eng.device, dtype=eng.dtype)
            for idx, name in enumerate(self.out_names):
                c = _lib.COMPONENTS[name]
                la[c, :, :, :W] = g[idx] if eng.is3d else g[idx].unsqueeze(0)
        # monitor DFT gradients: the same monitor structs with acc = dL/dF
        grads, mon_arr = [], (_lib.DnMonitor * max(1, len(eng.monitors)))()
        if eng.monitors:
            off = 0
            for m, spec in enumerate(eng.monitors):
                n = len(spec.wavelengths) * spec.cells * 2
                gm = (g_mon[off:off + n] if g_mon is not None
                      else torch.zeros(n, dtype=F64, device=eng.device))
                off += n
                gm = gm.to(device=eng.device, dtype=F64).contiguous()
                grads.append(gm)
                M = mon_arr[m]
                M.component = eng.mon_arr[m].component
                M.box = eng.mon_arr[m].box
                M.n_freq = eng.mon_arr[m].n_freq
                M.phase = eng.mon_arr[m].phase
                M.n_t = eng.mon_arr[m].n_t
                M.acc = gm.data_ptr()
        n_mon = len(eng.monitors) if g_mon is not None else 0
        grad_ce = torch.zeros((D, H, eng.Wp), dtype=F64, device=eng.device)
        T, K = eng.n_steps, self.K
        curl = eng.curl_buffer(min(K, T))
        starts = list(range(0, T, K))
        for ta in reversed(starts):
            tb = min(T, ta + K)
            # replay the segment from its checkpoint, recording the curls
            if ta == 0:
                eng.A.zero_()
                eng.B.zero_()
                eng.cur_b = False
            else:
                eng.cur_b = False
                eng.A.copy_(self.checkpoints[ta])
            rec = eng.curl_record(curl, ta, tb - ta)
            eng.run(ta, tb - ta, record=rec, outputs=False)
            ended_b = eng.adjoint(la, lb, rec, grad_ce, mon_arr, n_mon, tb, tb - ta)
            if ended_b:
                la, lb = lb, la
        eng.check_status(extra=(grad_ce[..., :W],))
        del grads
        return grad_ce[..., :W]


class _FDTDAdjoint(torch.autograd.Function):
    """Gradient of the FDTD outputs by the hand-written discrete adjoint."""

    @staticmethod
    def forward(ctx, eps, runner, save):
        eps_dev = eps.detach().to(runner.eng.device)
        field, mon = runner.forward(eps_dev, save)
        ctx.runner = runner
        ctx.save_for_backward(eps)
        return field, mon

    @staticmethod
    def backward(ctx, g_field, g_mon):
        (eps,) = ctx.saved_tensors
        runner = ctx.runner
        grad_ce = runner.adjoint(g_field, g_mon if g_mon is not None and g_mon.numel() else None)
        e = eps.detach().to(device=grad_ce.device, dtype=F64).reshape(grad_ce.shape)
        g = -(runner.eng.dt / (e * e)) * grad_ce
        ctx.runner = None
        return g.reshape(eps.shape).to(device=eps.device, dtype=eps.dtype), None, None


class _TimeReversalFDTD(_FDTDAdjoint):
    """``backward="time_reversal"``: same adjoint kernels (named like the
    reference's ``_TimeReversalFDTD`` so its grad_fn is recognisable)."""


def run_forward(solver, eng, eps: torch.Tensor, out_names):
    """Run all steps; return (field, [monitor DFTs]) -- differentiable with
    respect to ``eps`` when it requires grad."""
    if isinstance(out_names, str):
        out_names = (out_names,)
    needs_grad = eps.requires_grad and torch.is_grad_enabled()
    interval = checkpoint_interval(eng.n_steps, solver.use_checkpoint or
                                   getattr(solver, "backward", "") == "checkpoint",
                                   solver.checkpoint_segments)
    runner = _Runner(eng, out_names, interval if needs_grad else eng.n_steps)
    if needs_grad:
        fn = _TimeReversalFDTD if getattr(solver, "backward", "auto") == "time_reversal" \
            else _FDTDAdjoint
        field, mon = fn.apply(eps, runner, True)
    else:
        with torch.no_grad():
            field, mon = runner.forward(eps.detach(), False)
    dfts = []
    off = 0
    for spec in eng.monitors:
        n = len(spec.wavelengths) * spec.cells * 2
        shape = spec.shape if eng.is3d else spec.shape[1:]
        dfts.append(torch.view_as_complex(mon[off:off + n].reshape(-1, 2))
                    .reshape(len(spec.wavelengths), *shape))
        off += n
    if len(out_names) == 1:
        field = field[0]
    return field, dfts
