"""Generate ``design_ref.npz``: outputs of DiffNano's own design-layer operators.

Run once, in a container that has the reference checkout (read-only); its
location comes from ``DIFFNANO_REFERENCE`` (default ``/root/reference``)::

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_design_golden.py

The reference's ``diffnano/design/__init__.py`` imports modules that need
packages absent here, so the three files whose operators define the design
inputs are loaded directly from their paths (each imports only torch):

* ``diffnano/design/projection.py`` -- ``smooth_filter``, ``heaviside_projection``,
  ``beta_continuation_schedule``;
* ``diffnano/design/constraints_shared/primitives.py`` -- ``minimum_cd_penalty``
  (its erosion / dilation pair, ``-max_pool2d(-x)`` then ``max_pool2d``);
* ``diffnano/design/parameterization.py`` -- ``DensityField.forward``.

All runs are FP64 on the CPU on seeded inputs; gradients come from autograd.
Nothing at test time reads the reference; ``tests/test_design_golden.py``
reads the file this writes.
"""

from __future__ import annotations

import importlib.util
import os

import numpy as np
import torch

REF = os.environ.get("DIFFNANO_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))

RADII = (0.5, 1.0, 2.0, 2.5, 3.0, 4.0, 6.0)
BETAS = (1.0, 3.0, 8.0, 32.0)
ETAS = (0.5, 0.3)
SCHEDULE = [(s, n, b0, b1) for n, b0, b1 in ((100, 1.0, 32.0), (500, 1.0, 64.0), (37, 2.0, 16.0))
            for s in (0, 1, 7, n // 3, n // 2, n - 1, n, n + 5)]
MIN_CD = (2.0, 3.0)  # r = max(1, int(c / 2)) = 1: the 3 x 3 erosion / dilation


def _load(rel: str, name: str):
    spec = importlib.util.spec_from_file_location(name, os.path.join(REF, rel))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main() -> None:
    proj = _load("diffnano/design/projection.py", "_ref_projection")
    prim = _load("diffnano/design/constraints_shared/primitives.py", "_ref_primitives")
    para = _load("diffnano/design/parameterization.py", "_ref_parameterization")
    g = torch.Generator().manual_seed(2024)
    x3 = torch.rand(3, 40, 36, dtype=torch.float64, generator=g)
    x2 = torch.rand(29, 33, dtype=torch.float64, generator=g)
    blobs = (torch.rand(2, 48, 48, dtype=torch.float64, generator=g) > 0.5).to(torch.float64)
    out = {"x3": x3.numpy(), "x2": x2.numpy(), "blobs": blobs.numpy(),
           "radii": np.array(RADII), "betas": np.array(BETAS), "etas": np.array(ETAS),
           "schedule_args": np.array(SCHEDULE, dtype=np.float64),
           "min_cd": np.array(MIN_CD)}
    for r in RADII:
        out[f"smooth3_r{r}"] = proj.smooth_filter(x3, radius=r).numpy()
        out[f"smooth2_r{r}"] = proj.smooth_filter(x2, radius=r).numpy()
    for b in BETAS:
        for e in ETAS:
            out[f"heaviside_b{b}_e{e}"] = proj.heaviside_projection(x3, beta=b, eta=e).numpy()
            df = para.DensityField(grid_shape=(40, 36), eps_low=2.085, eps_high=12.1, beta=b,
                                   eta=e)
            out[f"density_field_b{b}_e{e}"] = df.forward(x3[0]).numpy()
    out["schedule"] = np.array([proj.beta_continuation_schedule(int(s), int(n), b0, b1)
                                for s, n, b0, b1 in SCHEDULE])
    for c in MIN_CD:
        for name, x in (("x3", x3), ("blobs", blobs)):
            xx = x.clone().requires_grad_(True)
            p = prim.minimum_cd_penalty(xx, min_cd_pixels=c)
            p.backward()
            out[f"mincd_{name}_c{c}"] = np.array(float(p.detach()))
            out[f"mincd_grad_{name}_c{c}"] = xx.grad.numpy()
    np.savez_compressed(os.path.join(HERE, "design_ref.npz"), **out)
    print(f"wrote {len(out)} arrays to design_ref.npz")


if __name__ == "__main__":
    main()
