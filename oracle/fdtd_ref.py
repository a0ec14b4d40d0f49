"""CPU FP64 oracle for the differentiable Yee-FDTD path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``diffnano_b200``) imports
this module; only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` use it, and only as the checker / the timed CPU baseline.

What it is: a restatement, written for this project, of the arithmetic of
DiffNano's FDTD solvers (``diffnano/solvers/fdtd2d.py`` and
``diffnano/solvers/fdtd3d.py``), in FP64 on the CPU, using torch CPU tensors
as the array library (the same library and dtype the reference runs on, so
elementwise rounding is identical and the restatement is bit-exact against the
reference's own outputs; ``tests/test_oracle_golden.py`` pins that against the
fixtures in ``tests/golden/``).  Each function cites the reference lines it
follows.  The operation order inside each update expression is kept the same
as the reference's on purpose: it is what makes the FP64 results bit-exact.

Gradients come from torch autograd through this restatement, which is exactly
the reference's own gradient algorithm (``backward="auto"`` is plain autograd;
``backward="time_reversal"`` re-runs the forward with autograd,
``fdtd3d.py:184-217``).

Extensions that the reference lacks (Ex/Ey/Hx/Hy source components, DFT
monitors, the figure of merit, the ``"physical"`` 3-D CPML axis mapping) are
defined here in the same style and are the oracle for the CUDA kernels'
extensions.
"""

from __future__ import annotations

import math

import torch

F64 = torch.float64

__all__ = [
    "cpml_profile",
    "waveform",
    "waveform_table",
    "source_box_2d",
    "source_box_3d",
    "box_mask",
    "step_tm",
    "step_te",
    "step_3d",
    "run_2d",
    "run_3d",
    "dft_phase",
    "fom_abs2",
]


# ---------------------------------------------------------------------------
# a1: CPML damping profile
# ---------------------------------------------------------------------------


def cpml_profile(size: int, pml_layers: int, dl: float, dt: float,
                 sigma_max: float = 0.8, order: int = 3):
    """1-D damping profile ``(b, c)`` of length ``size`` (FP64).

    Follows ``fdtd2d.py:67-88`` (identical to ``fdtd3d.py:66-85``): cubic
    grading sigma[i] = sigma_max*((L-i)/L)**order mirrored on both ends,
    sigma_s = sigma*dl/dt, alpha = 0.02*sigma_s, b = exp(-(sigma_s+alpha)*dt),
    c = sigma_s*(b-1)/(sigma_s+alpha+1e-30) where sigma_s+alpha > 1e-30 else 0.
    (The reference also builds a kappa array that it never uses.)
    """
    sigma = torch.zeros(size, dtype=F64)
    if pml_layers > 0:
        for i in range(pml_layers):
            d = (pml_layers - i) / pml_layers
            val = sigma_max * d ** order
            sigma[i] = val
            sigma[size - 1 - i] = val
    s = sigma * dl / dt
    alpha = 0.02 * s
    b = torch.exp(-(s + alpha) * dt)
    c = torch.where(s + alpha > 1e-30, s * (b - 1.0) / (s + alpha + 1e-30),
                    torch.zeros_like(s))
    return b, c


# ---------------------------------------------------------------------------
# a2: source waveform
# ---------------------------------------------------------------------------


def waveform(step: int, dt: float, omega: float, source: dict) -> float:
    """Source amplitude at ``step`` (FP64 value; its sine is FP32).

    Follows ``fdtd2d.py:178-205`` / ``fdtd3d.py:319-338``.  For the Gaussian
    pulse the sine's argument ``omega*t`` is rounded to FP32 and the sine is
    evaluated in FP32 (the reference builds that tensor with the default
    dtype), ``amp*sin`` is an FP32 product, and the envelope is FP64.  The
    "continuous" source is pure Python FP64.  Any other type gives 0.
    """
    kind = source.get("type", "gaussian_pulse")
    t = step * dt
    if kind == "gaussian_pulse":
        t0 = source.get("t0", 3.0 / omega)
        spread = source.get("spread", 1.0 / omega)
        amp = source.get("amplitude", 1.0)
        t_t = torch.tensor(t, dtype=F64)
        t0_t = torch.tensor(t0, dtype=F64)
        spread_t = torch.tensor(spread, dtype=F64)
        sin_val = torch.sin(torch.tensor(omega * t, dtype=torch.float32))
        env = torch.exp(-((t_t - t0_t) ** 2) / (2 * spread_t ** 2))
        return float(amp * sin_val * env)
    if kind == "continuous":
        amp = source.get("amplitude", 1.0)
        ramp = min(1.0, t * omega / (4 * math.pi))
        return float(amp * ramp * math.sin(omega * t))
    return 0.0


def waveform_table(n_steps: int, dt: float, omega: float, source: dict,
                   t_start: int = 0) -> torch.Tensor:
    """``waveform`` for steps ``t_start .. t_start+n_steps-1`` (FP64 tensor)."""
    return torch.tensor([waveform(t_start + s, dt, omega, source) for s in range(n_steps)],
                        dtype=F64)


# ---------------------------------------------------------------------------
# a3: source placement (as index boxes) and masks
# ---------------------------------------------------------------------------


def source_box_2d(shape, source: dict):
    """Index box ``((i0, i1), (j0, j1))`` the reference's 2-D mask covers.

    Follows ``fdtd2d.py:207-227``: ``pos=[y, x]`` gives one cell, otherwise
    ``row`` (default H//2) gives a full row; out-of-range positions give an
    empty mask (returned as ``None``).
    """
    H, W = shape
    pos = source.get("pos", None)
    if pos is not None:
        y, x = pos
        if 0 <= y < H and 0 <= x < W:
            return ((y, y + 1), (x, x + 1))
        return None
    row = source.get("row", H // 2)
    if 0 <= row < H:
        return ((row, row + 1), (0, W))
    return None


def source_box_3d(shape, source: dict):
    """Index box ``((i0,i1),(j0,j1),(k0,k1))`` of the reference's 3-D mask.

    Follows ``fdtd3d.py:340-372``: ``pos=[z,y,x]`` one cell; ``plane`` "xy"
    (at ``z``, default D//2), "xz" (at ``y``), "yz" (at ``x``); otherwise the
    line ``[D//2, H//2, :]``.  Out-of-range gives ``None``.
    """
    D, H, W = shape
    pos = source.get("pos", None)
    if pos is not None:
        z, y, x = pos
        if 0 <= z < D and 0 <= y < H and 0 <= x < W:
            return ((z, z + 1), (y, y + 1), (x, x + 1))
        return None
    plane = source.get("plane", None)
    if plane == "xy":
        z = source.get("z", D // 2)
        return ((z, z + 1), (0, H), (0, W)) if 0 <= z < D else None
    if plane == "xz":
        y = source.get("y", H // 2)
        return ((0, D), (y, y + 1), (0, W)) if 0 <= y < H else None
    if plane == "yz":
        x = source.get("x", W // 2)
        return ((0, D), (0, H), (x, x + 1)) if 0 <= x < W else None
    return ((D // 2, D // 2 + 1), (H // 2, H // 2 + 1), (0, W))


def box_mask(shape, box) -> torch.Tensor:
    """Dense FP64 0/1 mask of ``box`` (``None`` gives all zeros)."""
    m = torch.zeros(*shape, dtype=F64)
    if box is not None:
        m[tuple(slice(a, b) for a, b in box)] = 1.0
    return m


# ---------------------------------------------------------------------------
# a4/a5: 2-D leapfrog steps
# ---------------------------------------------------------------------------


def _dfwd(f, axis):
    """Forward difference f[a+1]-f[a] along ``axis`` with the last index 0."""
    d = torch.zeros_like(f)
    n = f.shape[axis]
    hi = [slice(None)] * f.dim()
    lo = [slice(None)] * f.dim()
    hi[axis] = slice(1, n)
    lo[axis] = slice(0, n - 1)
    d[tuple(lo)] = f[tuple(hi)] - f[tuple(lo)]
    return d


def _dbwd(f, axis):
    """Backward difference f[a]-f[a-1] along ``axis`` with the first index 0."""
    d = torch.zeros_like(f)
    n = f.shape[axis]
    hi = [slice(None)] * f.dim()
    lo = [slice(None)] * f.dim()
    hi[axis] = slice(1, n)
    lo[axis] = slice(0, n - 1)
    d[tuple(hi)] = f[tuple(hi)] - f[tuple(lo)]
    return d


def step_tm(Ez, Hx, Hy, eps, prof, dt, dl):
    """One TMz step (no source).  Follows ``fdtd2d.py:233-267``.

    ``prof = (b_x, c_x, b_y, c_y)``: x-profiles have length W and index the
    column j, y-profiles have length H and index the row i.  Hx is damped by
    the row profile while its difference runs along j; Hy the other way round.
    """
    bx, cx, by, cy = prof
    bxr, cxr = bx.unsqueeze(0), cx.unsqueeze(0)
    byc, cyc = by.unsqueeze(1), cy.unsqueeze(1)
    dEz_j = _dfwd(Ez, 1) / dl
    Hx = byc * Hx - dt * (cyc * dEz_j + dEz_j)
    dEz_i = _dfwd(Ez, 0) / dl
    Hy = bxr * Hy + dt * (cxr * dEz_i + dEz_i)
    dHy_i = _dbwd(Hy, 0) / dl
    dHx_j = _dbwd(Hx, 1) / dl
    Ez = bxr * byc * Ez + (dt / eps) * (cxr * dHy_i + dHy_i - cyc * dHx_j - dHx_j)
    return Ez, Hx, Hy


def step_te(Hz, Ex, Ey, eps, prof, dt, dl):
    """One TE step (no source).  Follows ``fdtd2d.py:269-303``."""
    bx, cx, by, cy = prof
    bxr, cxr = bx.unsqueeze(0), cx.unsqueeze(0)
    byc, cyc = by.unsqueeze(1), cy.unsqueeze(1)
    dHz_j = _dbwd(Hz, 1) / dl
    Ex = bxr * Ex + (dt / eps) * (cxr * dHz_j + dHz_j)
    dHz_i = _dbwd(Hz, 0) / dl
    Ey = byc * Ey - (dt / eps) * (cyc * dHz_i + dHz_i)
    dEy_i = _dfwd(Ey, 0) / dl
    dEx_j = _dfwd(Ex, 1) / dl
    Hz = bxr * byc * Hz + dt * (cxr * dEy_i + dEy_i - cyc * dEx_j - dEx_j)
    return Hz, Ex, Ey


# ---------------------------------------------------------------------------
# a6: 3-D step
# ---------------------------------------------------------------------------


def _coef3d(prof, axes):
    """Broadcast views of the six 1-D profiles for one axis mapping.

    ``prof = (b_x, c_x, b_y, c_y, b_z, c_z)`` with x = W (index k), y = H
    (index j), z = D (index i).

    ``axes="reference"`` reproduces the reference's broadcasting exactly
    (``fdtd3d.py:402-463``): ``b_y, c_y`` index j; ``b_z, c_z`` index k;
    ``b_x`` indexes k in Hz/Ez and j in Ey; ``c_x`` indexes j in Hy/Ey and k
    in Hz/Ez.  It only broadcasts on cubic grids, like the reference.

    ``axes="physical"`` indexes every profile along its own named axis (the
    reference's evident intent), which works on any (D, H, W).
    """
    bx, cx, by, cy, bz, cz = prof
    at_i = lambda v: v.view(-1, 1, 1)  # noqa: E731
    at_j = lambda v: v.view(1, -1, 1)  # noqa: E731
    at_k = lambda v: v.view(1, 1, -1)  # noqa: E731
    if axes == "reference":
        return dict(
            hx_b=at_j(by), hx_c1=at_j(cy), hx_c2=at_k(cz),
            hy_b=at_k(bz), hy_c1=at_k(cz), hy_c2=at_j(cx),
            hz_b=at_k(bx), hz_c1=at_k(cx), hz_c2=at_j(cy),
            ex_b1=at_j(by), ex_b2=at_k(bz), ex_c1=at_j(cy), ex_c2=at_k(cz),
            ey_b1=at_k(bz), ey_b2=at_j(bx), ey_c1=at_k(cz), ey_c2=at_j(cx),
            ez_b1=at_k(bx), ez_b2=at_j(by), ez_c1=at_k(cx), ez_c2=at_j(cy),
        )
    if axes == "physical":
        return dict(
            hx_b=at_j(by), hx_c1=at_j(cy), hx_c2=at_i(cz),
            hy_b=at_i(bz), hy_c1=at_i(cz), hy_c2=at_k(cx),
            hz_b=at_k(bx), hz_c1=at_k(cx), hz_c2=at_j(cy),
            ex_b1=at_j(by), ex_b2=at_i(bz), ex_c1=at_j(cy), ex_c2=at_i(cz),
            ey_b1=at_i(bz), ey_b2=at_k(bx), ey_c1=at_i(cz), ey_c2=at_k(cx),
            ez_b1=at_k(bx), ez_b2=at_j(by), ez_c1=at_k(cx), ez_c2=at_j(cy),
        )
    raise ValueError(f"unknown cpml axes {axes!r}")


def step_3d(Ex, Ey, Ez, Hx, Hy, Hz, eps, prof, dt, dl, axes="reference"):
    """One 3-D Yee step, H from old E then E from new H (no source).

    Follows ``fdtd3d.py:378-465`` term by term (axis 0 = z = i, 1 = y = j,
    2 = x = k; forward differences zero at the last index, backward
    differences zero at the first).
    """
    q = _coef3d(prof, axes)
    dEz_y = _dfwd(Ez, 1) / dl
    dEy_z = _dfwd(Ey, 0) / dl
    Hx = q["hx_b"] * Hx - dt * (q["hx_c1"] * dEz_y + dEz_y - q["hx_c2"] * dEy_z - dEy_z)
    dEx_z = _dfwd(Ex, 0) / dl
    dEz_x = _dfwd(Ez, 2) / dl
    Hy = q["hy_b"] * Hy - dt * (q["hy_c1"] * dEx_z + dEx_z - q["hy_c2"] * dEz_x - dEz_x)
    dEy_x = _dfwd(Ey, 2) / dl
    dEx_y = _dfwd(Ex, 1) / dl
    Hz = q["hz_b"] * Hz - dt * (q["hz_c1"] * dEy_x + dEy_x - q["hz_c2"] * dEx_y - dEx_y)

    ce = dt / eps
    dHz_y = _dbwd(Hz, 1) / dl
    dHy_z = _dbwd(Hy, 0) / dl
    Ex = q["ex_b1"] * q["ex_b2"] * Ex + ce * (
        q["ex_c1"] * dHz_y + dHz_y - q["ex_c2"] * dHy_z - dHy_z)
    dHx_z = _dbwd(Hx, 0) / dl
    dHz_x = _dbwd(Hz, 2) / dl
    Ey = q["ey_b1"] * q["ey_b2"] * Ey + ce * (
        q["ey_c1"] * dHx_z + dHx_z - q["ey_c2"] * dHz_x - dHz_x)
    dHy_x = _dbwd(Hy, 2) / dl
    dHx_y = _dbwd(Hx, 1) / dl
    Ez = q["ez_b1"] * q["ez_b2"] * Ez + ce * (
        q["ez_c1"] * dHy_x + dHy_x - q["ez_c2"] * dHx_y - dHx_y)
    return Ex, Ey, Ez, Hx, Hy, Hz


# ---------------------------------------------------------------------------
# a12: DFT monitors and the figure of merit (extensions; no reference code)
# ---------------------------------------------------------------------------


def dft_phase(n_steps: int, dt: float, wavelengths_nm) -> torch.Tensor:
    """Phase table ``(T, L, 2)``: (cos(w t_n)*dt, -sin(w t_n)*dt), t_n = n*dt.

    A monitor's DFT is F(r) = sum_n f_n(r) * exp(-i*w*t_n) * dt, where f_n is
    the field after step n (source already injected) -- the same sample the
    reference's ``time_series`` records at index n (``fdtd2d.py:335-337``).
    """
    out = torch.zeros(n_steps, len(wavelengths_nm), 2, dtype=F64)
    for li, lam in enumerate(wavelengths_nm):
        w = 2.0 * math.pi / lam
        for n in range(n_steps):
            out[n, li, 0] = math.cos(w * n * dt) * dt
            out[n, li, 1] = -math.sin(w * n * dt) * dt
    return out


def fom_abs2(dft: torch.Tensor) -> torch.Tensor:
    """Figure of merit sum |F|^2 of a ``(..., 2)`` (re, im) DFT tensor."""
    return (dft[..., 0] ** 2 + dft[..., 1] ** 2).sum()


# ---------------------------------------------------------------------------
# a7/a11: run loops
# ---------------------------------------------------------------------------


def _monitor_slices(mon):
    return tuple(slice(a, b) for a, b in mon["box"])


def run_2d(eps, *, dl, dt, omega, pml_layers, polarization="TM", n_steps, source,
           monitors=(), probe=None, component=None):
    """Run the 2-D solver from zero fields; follows ``fdtd2d.py:309-357``.

    ``source`` is the reference's source dict; its mask comes from
    ``source_box_2d``.  The injected field is Ez (TM) / Hz (TE) as in the
    reference (``fdtd2d.py:333,351``).  ``monitors`` is a list of dicts with
    ``component``, ``box`` (index box) and ``wavelengths_nm``.  Returns a dict
    with the final fields, the probe series (``fdtd2d.py:335-337``) and the
    monitor DFTs (each ``(L, *box_shape, 2)``).
    """
    H, W = eps.shape
    prof = (*cpml_profile(W, pml_layers, dl, dt), *cpml_profile(H, pml_layers, dl, dt))
    mask = box_mask((H, W), source_box_2d((H, W), source))
    f = {k: torch.zeros(H, W, dtype=F64) for k in ("Ez", "Hx", "Hy", "Hz", "Ex", "Ey")}
    phases = [dft_phase(n_steps, dt, m["wavelengths_nm"]) for m in monitors]
    acc = [None] * len(monitors)
    series = []
    for step in range(n_steps):
        w = waveform(step, dt, omega, source)
        if polarization == "TM":
            f["Ez"], f["Hx"], f["Hy"] = step_tm(f["Ez"], f["Hx"], f["Hy"], eps, prof, dt, dl)
            f["Ez"] = f["Ez"] + mask * w
            probe_field = f["Ez"]
        else:
            f["Hz"], f["Ex"], f["Ey"] = step_te(f["Hz"], f["Ex"], f["Ey"], eps, prof, dt, dl)
            f["Hz"] = f["Hz"] + mask * w
            probe_field = f["Hz"]
        if probe is not None:
            series.append(probe_field[probe[0], probe[1]].clone())
        for mi, m in enumerate(monitors):
            v = f[m["component"]][_monitor_slices(m)]
            ph = phases[mi][step]
            term = torch.stack([v.unsqueeze(0) * ph[:, 0].view(-1, *([1] * v.dim())),
                                v.unsqueeze(0) * ph[:, 1].view(-1, *([1] * v.dim()))], dim=-1)
            acc[mi] = term if acc[mi] is None else acc[mi] + term
    out = dict(f)
    out["series"] = torch.stack(series) if series else None
    out["monitors"] = acc
    return out


def run_3d(eps, *, dl, dt, omega, pml_layers, n_steps, source, monitors=(), probe=None,
           axes="reference", component="Ez", init=None, t0=0):
    """Run the 3-D solver; follows ``fdtd3d.py:471-504``.

    The reference starts from zero fields at step 0 and injects into Ez
    (``fdtd3d.py:502``); ``component`` selects Ex/Ey/Ez (extension).
    ``init`` (a dict of the six ``(D, H, W)`` fields) and ``t0`` start the
    loop from a given state at absolute step ``t0`` instead (extension: it
    lets a short run touch every cell of a large grid); the waveform and the
    DFT phases are taken at the absolute step, and monitors accumulate from
    ``t0``.  Returns a dict with the six final fields, the probe series of Ez
    (``fdtd3d.py:698``) and the monitor DFTs.
    """
    D, H, W = eps.shape
    prof = (*cpml_profile(W, pml_layers, dl, dt), *cpml_profile(H, pml_layers, dl, dt),
            *cpml_profile(D, pml_layers, dl, dt))
    mask = box_mask((D, H, W), source_box_3d((D, H, W), source))
    names = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
    if init is None:
        f = {k: torch.zeros(D, H, W, dtype=F64) for k in names}
    else:
        f = {k: init[k].to(F64).clone() for k in names}
    phases = [dft_phase(t0 + n_steps, dt, m["wavelengths_nm"]) for m in monitors]
    acc = [None] * len(monitors)
    series = []
    for step in range(t0, t0 + n_steps):
        new = step_3d(*(f[k] for k in names), eps, prof, dt, dl, axes=axes)
        f = dict(zip(names, new))
        w = waveform(step, dt, omega, source)
        f[component] = f[component] + mask * w
        if probe is not None:
            series.append(f["Ez"][probe[0], probe[1], probe[2]].clone())
        for mi, m in enumerate(monitors):
            v = f[m["component"]][_monitor_slices(m)]
            ph = phases[mi][step]
            shp = [-1] + [1] * v.dim()
            term = torch.stack([v.unsqueeze(0) * ph[:, 0].view(shp),
                                v.unsqueeze(0) * ph[:, 1].view(shp)], dim=-1)
            acc[mi] = term if acc[mi] is None else acc[mi] + term
    out = dict(f)
    out["series"] = torch.stack(series) if series else None
    out["monitors"] = acc
    return out
