"""Forward driver and (later) the autograd bridge for the FDTD kernels."""

from __future__ import annotations

import torch

from diffnano_b200 import _lib


def _outputs(eng, out_names):
    comps = [_lib.COMPONENTS[n] for n in out_names]
    f = torch.stack([eng.field(c)[0] if not eng.is3d else eng.field(c) for c in comps])
    dfts = [eng.monitor_dft(m).clone() for m in range(len(eng.monitors))]
    return f, dfts


def run_forward(solver, eng, eps: torch.Tensor, out_names):
    """Run all steps; return (field stack, [monitor DFTs])."""
    if isinstance(out_names, str):
        out_names = (out_names,)
    needs_grad = eps.requires_grad and torch.is_grad_enabled()
    if needs_grad:
        raise NotImplementedError("gradients: adjoint kernels not built yet")
    with torch.no_grad():
        eng.set_eps(eps.detach())
        eng.run(0, eng.n_steps)
        f, dfts = _outputs(eng, out_names)
    eng.check_status()
    if len(out_names) == 1:
        f = f[0]
    return f, dfts
