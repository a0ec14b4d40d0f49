"""Host-side set-up for the FDTD kernels: CPML profiles, source waveform
tables, source/monitor index boxes and DFT phase tables.

All of this is computed once per ``forward`` on the CPU in FP64 (O(T) or
O(N^(1/3)) values) and uploaded; none of it is on the per-step path.
"""

from __future__ import annotations

import math
from collections.abc import Sequence

import numpy as np
import torch

from diffnano_b200 import _lib

F64 = torch.float64


def cpml_profile(size: int, pml_layers: int, dl: float, dt: float,
                 sigma_max: float = 0.8, order: int = 3):
    """``(b, c)`` FP64 damping profile of one axis.

    Same arithmetic as ``_CPMLRegion`` (``diffnano/solvers/fdtd2d.py:67-88``,
    ``fdtd3d.py:66-85``): sigma = sigma_max*((L-i)/L)**3 mirrored,
    sigma_s = sigma*dl/dt, alpha = 0.02 sigma_s, b = exp(-(sigma_s+alpha) dt),
    c = sigma_s (b-1)/(sigma_s+alpha+1e-30) where sigma_s+alpha > 1e-30, else 0.
    """
    sigma = torch.zeros(size, dtype=F64)
    for i in range(max(0, pml_layers)):
        val = sigma_max * ((pml_layers - i) / pml_layers) ** order
        sigma[i] = val
        sigma[size - 1 - i] = val
    s = sigma * dl / dt
    a = 0.02 * s
    b = torch.exp(-(s + a) * dt)
    c = torch.where(s + a > 1e-30, s * (b - 1.0) / (s + a + 1e-30), torch.zeros_like(s))
    return b, c


def waveform_table(n_steps: int, dt: float, omega: float, source: dict) -> torch.Tensor:
    """Source amplitude for steps 0..n_steps-1 as an FP64 CPU tensor.

    Same expression as ``_source_waveform`` (``fdtd2d.py:178-205``,
    ``fdtd3d.py:319-338``), vectorised: for the Gaussian pulse the sine of
    the FP32-rounded argument is evaluated in FP32 and ``amp*sin`` is an FP32
    product, times the FP64 envelope; "continuous" is FP64 with a linear
    ramp over two periods; any other type is zero.
    """
    kind = source.get("type", "gaussian_pulse")
    steps = np.arange(n_steps, dtype=np.float64)
    t = steps * dt
    if kind == "gaussian_pulse":
        t0 = float(source.get("t0", 3.0 / omega))
        spread = float(source.get("spread", 1.0 / omega))
        amp = source.get("amplitude", 1.0)
        arg = torch.from_numpy(omega * t).to(torch.float32)
        s = amp * torch.sin(arg)
        env = torch.exp(-((torch.from_numpy(t) - t0) ** 2) / (2 * spread ** 2))
        return s.to(F64) * env
    if kind == "continuous":
        amp = float(source.get("amplitude", 1.0))
        vals = [amp * min(1.0, tt * omega / (4 * math.pi)) * math.sin(omega * tt) for tt in t.tolist()]
        return torch.tensor(vals, dtype=F64)
    return torch.zeros(n_steps, dtype=F64)


def source_box_2d(shape, source: dict):
    """Cells the reference's 2-D mask covers, as ``((0,1),(i0,i1),(j0,j1))``.

    ``fdtd2d.py:207-227``: ``pos=[y, x]`` is one cell; otherwise ``row``
    (default H//2) is a full row.  Out-of-range positions inject nothing
    (``None``), exactly as the reference silently does.
    """
    H, W = shape
    pos = source.get("pos", None)
    if pos is not None:
        y, x = int(pos[0]), int(pos[1])
        return ((0, 1), (y, y + 1), (x, x + 1)) if 0 <= y < H and 0 <= x < W else None
    row = int(source.get("row", H // 2))
    return ((0, 1), (row, row + 1), (0, W)) if 0 <= row < H else None


def source_box_3d(shape, source: dict):
    """Cells of the reference's 3-D mask (``fdtd3d.py:340-372``).

    ``pos=[z, y, x]``; ``plane`` "xy"/"xz"/"yz" at ``z``/``y``/``x``
    (default mid-plane); otherwise the x-line at (D//2, H//2).  Out of range:
    ``None`` (no injection).
    """
    D, H, W = shape
    pos = source.get("pos", None)
    if pos is not None:
        z, y, x = (int(v) for v in pos)
        ok = 0 <= z < D and 0 <= y < H and 0 <= x < W
        return ((z, z + 1), (y, y + 1), (x, x + 1)) if ok else None
    plane = source.get("plane", None)
    if plane == "xy":
        z = int(source.get("z", D // 2))
        return ((z, z + 1), (0, H), (0, W)) if 0 <= z < D else None
    if plane == "xz":
        y = int(source.get("y", H // 2))
        return ((0, D), (y, y + 1), (0, W)) if 0 <= y < H else None
    if plane == "yz":
        x = int(source.get("x", W // 2))
        return ((0, D), (0, H), (x, x + 1)) if 0 <= x < W else None
    return ((D // 2, D // 2 + 1), (H // 2, H // 2 + 1), (0, W))


def component_id(name: str, allowed: Sequence[str]) -> int:
    if name not in allowed:
        raise ValueError(f"field component {name!r} not available here; expected one of {list(allowed)}")
    return _lib.COMPONENTS[name]


def _check_box(box, shape3):
    for (a, b), n in zip(box, shape3):
        if not (0 <= a < b <= n):
            raise ValueError(f"monitor box {box} outside the grid {tuple(shape3)}")
    return tuple((int(a), int(b)) for a, b in box)


def monitor_box(spec: dict, shape3, is3d: bool):
    """Index box of a monitor spec.

    2-D keys: ``box=[[y0,y1],[x0,x1]]``, ``pos=[y,x]``, ``row=r`` (a full
    row) or ``col=c`` (a full column).  3-D keys: ``box=[[z0,z1],[y0,y1],
    [x0,x1]]``, ``pos=[z,y,x]``, or ``plane`` "xy"/"xz"/"yz" with ``z``/``y``/
    ``x`` and an optional in-plane ``extent=[[a0,a1],[b0,b1]]`` (the two
    in-plane axes in (z, y, x) order).  Out-of-range boxes raise ValueError.
    """
    D, H, W = shape3
    if "box" in spec:
        b = [list(v) for v in spec["box"]]
        if not is3d:
            b = [[0, 1]] + b
        return _check_box(b, shape3)
    if "pos" in spec:
        p = list(spec["pos"])
        if not is3d:
            p = [0] + p
        return _check_box([[v, v + 1] for v in p], shape3)
    if not is3d:
        if "row" in spec:
            r = int(spec["row"])
            return _check_box([[0, 1], [r, r + 1], [0, W]], shape3)
        if "col" in spec:
            c = int(spec["col"])
            return _check_box([[0, 1], [0, H], [c, c + 1]], shape3)
        raise ValueError(f"2-D monitor needs box/pos/row/col: {spec}")
    plane = spec.get("plane")
    full = [[0, D], [0, H], [0, W]]
    axis = {"xy": 0, "xz": 1, "yz": 2}.get(plane)
    if axis is None:
        raise ValueError(f"3-D monitor needs box/pos/plane: {spec}")
    at = int(spec.get("zyx"[axis], shape3[axis] // 2))
    full[axis] = [at, at + 1]
    if "extent" in spec:
        others = [a for a in range(3) if a != axis]
        for a, rng in zip(others, spec["extent"]):
            full[a] = list(rng)
    return _check_box(full, shape3)


def dft_phase_table(n_steps: int, dt: float, wavelengths_nm) -> torch.Tensor:
    """``(T, L, 2)`` FP64: ``(cos(w t_n) dt, -sin(w t_n) dt)`` with t_n = n dt.

    A monitor's DFT is F(r) = sum_n f_n(r) exp(-i w t_n) dt where f_n is the
    field after step n, source included -- the value ``time_series`` reports
    at index n.
    """
    w = 2.0 * np.pi / np.asarray(wavelengths_nm, dtype=np.float64)
    t = np.arange(n_steps, dtype=np.float64) * dt
    ph = np.outer(t, w)
    out = np.stack([np.cos(ph) * dt, -np.sin(ph) * dt], axis=-1)
    return torch.from_numpy(np.ascontiguousarray(out))
