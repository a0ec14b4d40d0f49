#!/usr/bin/env python
"""FDTD benchmark: 3-D 256^3 FP32 Yee step with CPML on B200.

Workload (one "step" = one leapfrog time step of the whole grid, H then E,
soft-source injection and a running-DFT monitor, all in the fused
``dn_fdtd3d_run`` kernel): 256^3 cells, dl = 25 nm, 12-cell CPML, Courant
0.4, FP32; eps = SiO2 substrate / 500 nm Si slab / air with a 128x128x40
design block of seeded filtered noise in [2.085, 12.1]; Ex-polarised
Gaussian-pulse plane source at 1.55 um; Ey DFT monitor on a 64x64 plane.
Inputs are synthetic (seeded), the state (2 x 6 x 67 MB + 67 MB) is larger
than the 126 MB L2, so no flush is needed between steps.

Prints one JSON line (rank 0).  ``--impl reference`` times the CPU FP64
restatement of the reference's algorithm (the oracle) on the host cores on
the same grid instead.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SHAPE = (256, 256, 256)
DL, COURANT, PML, T_SOLVE = 25.0, 0.4, 12, 4000
Z_SRC = 40
BYTES_PER_CELL_STEP = 52  # FP32: read Ex Ey Ez Hx Hy Hz dt/eps, write the six fields
# reverse step, algorithmic: forward recompute 52 + adjoint update 52 + dL/deps
# read-modify-write 8 (FP32)
ADJ_BYTES_PER_CELL_STEP = 112
# what the reverse step moves on top: the curl record written by the replay and
# read back by the adjoint (12 + 12) and the FP64 gradient's extra 8 bytes
ADJ_OVERHEAD_BYTES_PER_CELL_STEP = {"curl_record": 24, "fp64_gradient": 8}
WORKLOAD = "3d_yee_256cube_cpml12_fp32"
METRIC = "FDTD Gcell-updates/s"
UNIT = "Gcell-updates/s"


def fwd_kernel_name() -> str:
    """The FP32 3-D step kernel the library runs (two columns per lane unless
    DN_FDTD3D_LANE_COLUMNS=1 asks for the one-column kernel)."""
    return "k_fdtd3d" if os.environ.get("DN_FDTD3D_LANE_COLUMNS") == "1" else "k_fdtd3d_v2"


def workload():
    """eps, source dict and monitor spec of the cubic grid SHAPE."""
    from diffnano_b200.workloads import gaussian_pulse_for_band, slab_eps_3d

    n = SHAPE[0]
    eps = slab_eps_3d(SHAPE, dl=DL, design=(40, 128, 128), seed=1)
    src = gaussian_pulse_for_band(1550.0, 200.0)
    src.update(plane="xy", z=Z_SRC, component="Ex")
    c = n // 2
    mons = [{"name": "out", "component": "Ey", "plane": "xy", "z": n - 56,
             "extent": [[c - 32, c + 32], [c - 32, c + 32]], "wavelengths_nm": [1550.0]}]
    return eps, src, mons


def config_dict(extra=None):
    c = {"workload": WORKLOAD if SHAPE[0] == 256 else f"3d_yee_{SHAPE[0]}cube_cpml12_fp32",
         "grid": list(SHAPE), "dl_nm": DL, "pml_layers": PML,
         "courant": COURANT, "n_steps_per_solve": T_SOLVE,
         "source": "Ex plane-wave Gaussian pulse, 1550 nm, 200 nm band, plane z=40",
         "monitor": f"Ey DFT on a 64x64 plane at z={SHAPE[0] - 56}, 1550 nm",
         "l2": "inputs larger than L2 (state 940 MB ping-pong + 67 MB coefficients)",
         "parallelism": "replicas (one independent grid per GPU)"}
    if extra:
        c.update(extra)
    return c


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_per_launch():
    p = os.path.join(ROOT, "profiles", "fdtd3d_256_traffic.json")
    try:
        with open(p) as fh:
            return float(json.load(fh)["dram_bytes_per_launch"])
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock/throttle sampling (query only) in a reader thread.

    The 3-D timed window is only a few milliseconds, shorter than the 100 ms
    sampling period, so the caller starts the sampler, waits for its first
    sample (``wait_ready``) and keeps it running over the untimed pre-roll
    and the timed steps of the same solve: the summary is the clock under
    that load."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []
        self._thread = None

    def __enter__(self):
        import threading

        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.idx)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return self

        def reader():
            for ln in self.proc.stdout:
                if ln.strip():
                    self.lines.append(ln)

        self._thread = threading.Thread(target=reader, daemon=True)
        self._thread.start()
        return self

    def wait_ready(self, timeout: float = 5.0) -> None:
        t = time.perf_counter()
        while self.proc is not None and not self.lines and time.perf_counter() - t < timeout:
            time.sleep(0.01)

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            if self._thread is not None:
                self._thread.join(timeout=5)

    def summary(self, window: str | None = None):
        if not self.lines:
            return None
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        out = {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "samples": len(sm),
               "reasons": sorted(reasons)}
        if window:
            out["window"] = window
        return out


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, ws: int, dev) -> float:
    if ws == 1:
        return x
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rel_l2_dev(a, b) -> float:
    """Relative L2 error of ``a`` against ``b`` (real or complex; any device),
    computed in FP64 on ``b``'s device."""
    a = a.detach().to(b.device)
    if a.is_complex() or b.is_complex():
        a, b = torch.view_as_real(a.to(torch.complex128)), torch.view_as_real(b.to(torch.complex128))
    a, b = a.to(torch.float64), b.to(torch.float64)
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (FP64 torch CPU restatement of the reference)
# ---------------------------------------------------------------------------
def timed_window(K: int, Wm: int):
    """(pre-roll steps, total steps) of the 3-D timing: the K timed steps sit
    in the middle of a T_SOLVE-step solve, after Wm warm-up steps."""
    preroll = max(0, (T_SOLVE - K) // 2 - Wm)
    return preroll, max(T_SOLVE, preroll + Wm + K)


def oracle_sample(K: int, Wm: int, t_start: int):
    """Time K steps (after Wm warm-up steps) of the reference's algorithm on
    the host cores: the oracle (FP64 torch-CPU restatement of
    ``fdtd3d.py:_time_step`` + soft source, bit-exact with the reference) on
    the full 256^3 grid with the Ex plane source and the Ey DFT monitor, at
    absolute steps t_start .. t_start+K-1.  Returns (Gcell/s, seconds per
    step, description)."""
    from oracle import fdtd_ref as R

    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    eps, src, _ = workload()
    D, H, W = SHAPE
    dt = COURANT * DL / math.sqrt(3.0)
    c = D // 2
    mon = [{"component": "Ey", "box": ((D - 56, D - 55), (c - 32, c + 32), (c - 32, c + 32)),
            "wavelengths_nm": [1550.0]}]
    # the zero state at step t_start would need t_start CPU steps first (hours);
    # a seeded random state costs the same per step
    gen = torch.Generator().manual_seed(0)
    names = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
    state = {k: 1e-3 * torch.randn(D, H, W, dtype=torch.float64, generator=gen) for k in names}
    kw = dict(dl=DL, dt=dt, omega=2 * math.pi / 1550.0, pml_layers=PML, source=src,
              monitors=mon, component="Ex")
    if Wm:
        state = R.run_3d(eps, n_steps=Wm, init=state, t0=t_start - Wm, **kw)
    t = time.perf_counter()
    R.run_3d(eps, n_steps=K, init=state, t0=t_start, **kw)
    el = time.perf_counter() - t
    desc = (f"{K} time steps (after {Wm} warm-up steps) of the full 256^3 grid from a seeded "
            f"random state, steps {t_start}..{t_start + K - 1}: FP64 torch-CPU restatement of "
            "the reference's fdtd3d.py:_time_step with the Ex plane source and the Ey DFT "
            f"monitor (oracle/fdtd_ref.py), {threads} threads")
    return D * H * W * K / el / 1e9, el / K, desc, threads


def run_reference(args):
    """``--impl reference``: the CPU arm, on rank 0 only (see ``oracle_sample``);
    a long ``--steps`` is sampled by its first 100 steps (per-step cost is
    constant)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    K, Wm = args.steps, args.warmup
    preroll, _ = timed_window(K, Wm)
    t_start = preroll + Wm
    k_eff, w_eff = min(K, 100), min(Wm, 5)
    v, s_step, desc, threads = oracle_sample(k_eff, w_eff, t_start)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws,
            "steps": K, "warmup": Wm, "ms_per_step": s_step * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": config_dict({"timed_steps": [t_start, t_start + K]}),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": desc},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args):
    ws, rank, local = dist_setup()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    import diffnano_b200 as dn

    eps, src, mons = workload()
    D, H, W = SHAPE
    cells = D * H * W
    K, Wm = args.steps, args.warmup
    # The timed window sits in the middle of a T_SOLVE-step solve: once the pulse
    # fills the grid the board draws ~950 W and the power cap lowers the clocks,
    # so steps on a still mostly zero field are a few percent faster than the
    # solve's average.  Untimed pre-roll steps bring the state there first.
    preroll, n_total = timed_window(K, Wm)
    solver = dn.FDTDSolver3D(grid_shape=SHAPE, dl=DL, wavelength_nm=1550.0, pml_layers=PML,
                             n_steps=n_total, courant=COURANT, device=dev, dtype=torch.float32)
    eng = solver._make_engine(n_total, src, mons)
    eng.set_eps(eps.to(dev))
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as cs:
        cs.wait_ready()
        eng.run(0, preroll + Wm)
        torch.cuda.synchronize(dev)
        barrier(ws)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        eng.run(preroll + Wm, K)
        e1.record(stream)
        torch.cuda.synchronize(dev)
    barrier(ws)
    el = e0.elapsed_time(e1) / 1e3
    eng.check_status()
    el_max = max_over_ranks(el, ws, dev)
    value = ws * cells * K / el_max / 1e9
    launch_s = el / K
    peak, peak_kind = measured_peak_hbm()
    achieved = BYTES_PER_CELL_STEP * cells / launch_s / 1e9
    traffic = traffic_per_launch()
    del eng
    torch.cuda.empty_cache()

    # adjoint: reverse sweep (segment replay with curl record + reverse steps)
    adjoint = None
    if not args.no_adjoint:
        from diffnano_b200.solvers._adjoint import _Runner

        Ta = args.adjoint_steps
        eng_a = solver._make_engine(Ta, src, mons)
        runner = _Runner(eng_a, ("Ez", "Ex", "Ey"), int(math.ceil(math.sqrt(Ta))))
        with torch.no_grad():
            runner.forward(eps.to(dev), True)
        gen = torch.Generator(device=dev).manual_seed(0)
        g_field = torch.randn((3, D, H, W), device=dev, generator=gen)
        runner.adjoint(g_field, None)  # warm-up (also sizes the allocator's cache)
        torch.cuda.synchronize(dev)
        barrier(ws)
        e0.record(stream)
        runner.adjoint(g_field, None)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        el_a = max_over_ranks(e0.elapsed_time(e1) / 1e3, ws, dev)
        rev_s = el_a / Ta
        moved = ADJ_BYTES_PER_CELL_STEP + sum(ADJ_OVERHEAD_BYTES_PER_CELL_STEP.values())
        adjoint = {"value": ws * cells * Ta / el_a / 1e9, "unit": UNIT,
                   "ms_per_step": rev_s * 1e3, "steps": Ta,
                   "algorithmic_bytes_per_cell_step": ADJ_BYTES_PER_CELL_STEP,
                   "achieved_GBs": ADJ_BYTES_PER_CELL_STEP * cells / rev_s / 1e9,
                   "frac_of_hbm_peak": ADJ_BYTES_PER_CELL_STEP * cells / rev_s / 1e9 / peak,
                   "overhead_bytes_per_cell_step": ADJ_OVERHEAD_BYTES_PER_CELL_STEP,
                   "moved_GBs": moved * cells / rev_s / 1e9,
                   "what": f"reverse sweep of a {Ta}-step solve: per step one replay step with "
                           f"curl record ({fwd_kernel_name()}) + one reverse step (k_adj3d), "
                           f"checkpoints every {runner.K} steps"}
        del runner, eng_a
        torch.cuda.empty_cache()

    # end to end through the public API with host buffers (reference device="cpu")
    e2e = None
    if not args.no_e2e:
        s_host = dn.FDTDSolver3D(grid_shape=SHAPE, dl=DL, wavelength_nm=1550.0, pml_layers=PML,
                                 n_steps=T_SOLVE, courant=COURANT, device="cpu",
                                 dtype=torch.float32)
        eps_pinned = eps.to(torch.float32).pin_memory()
        # warm-up: two calls, since a loop that keeps its previous result while
        # the next one is made alternates between two page-locked result blocks
        # of torch's caching host allocator (the first use of each pays for the
        # page-locked allocation, ~0.1 s for the 201 MB field)
        for _ in range(2):
            r = s_host.forward(eps_pinned, source=dict(src), monitors=mons)
        barrier(ws)
        t = time.perf_counter()
        for _ in range(args.e2e_steps):
            r = s_host.forward(eps_pinned, source=dict(src), monitors=mons)
        e2e_el = (time.perf_counter() - t) / args.e2e_steps
        e2e_el = max_over_ranks(e2e_el, ws, dev)
        d2h = r.field.numel() * r.field.element_size() + sum(
            m["dft"].numel() * m["dft"].element_size() for m in r.metadata["monitors"])
        e2e = {"value": ws * cells * T_SOLVE / e2e_el / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": eps_pinned.numel() * eps_pinned.element_size(),
               "d2h_bytes_per_step": d2h,
               "step": f"one FDTDSolver3D.forward(device='cpu') solve of {T_SOLVE} time steps "
                       f"(host eps in, host field + monitor DFT out), mean of {args.e2e_steps}"}

    # the same 4000-step solve through the FP64 build of the kernels (untimed):
    # the error of the FP32 result that e2e timed
    fp64_check = None
    if not args.no_fp64_check and e2e is not None:
        s64 = dn.FDTDSolver3D(grid_shape=SHAPE, dl=DL, wavelength_nm=1550.0, pml_layers=PML,
                              n_steps=T_SOLVE, courant=COURANT, device=dev,
                              dtype=torch.float64)
        with torch.no_grad():
            r64 = s64.forward(eps.to(dev), source=dict(src), monitors=mons)
        fp64_check = {
            "field_rel_l2": rel_l2_dev(r.field, r64.field),
            "dft_rel_l2": rel_l2_dev(r.metadata["monitors"][0]["dft"],
                                     r64.metadata["monitors"][0]["dft"]),
            "what": f"FP32 result of the timed {T_SOLVE}-step solve vs the same solve on the "
                    "FP64 kernels: field [Ez, Ex, Ey] and Ey DFT, relative L2"}
        del r64, s64
        torch.cuda.empty_cache()

    # full gradient of the monitor FOM through the public API, host buffers
    grad_e2e = None
    if not args.no_grad_e2e:
        s_host = dn.FDTDSolver3D(grid_shape=SHAPE, dl=DL, wavelength_nm=1550.0, pml_layers=PML,
                                 n_steps=T_SOLVE, courant=COURANT, device="cpu",
                                 dtype=torch.float32, backward="time_reversal")
        # one untimed call first (checkpoint buffers and the allocator's first
        # growth), as the forward e2e leg does
        e_in = eps.to(torch.float32).pin_memory().requires_grad_(True)
        r = s_host.forward(e_in, source=dict(src), monitors=mons)
        (r.metadata["monitors"][0]["dft"].abs() ** 2).sum().backward()
        del r
        e_in = eps.to(torch.float32).pin_memory().requires_grad_(True)
        barrier(ws)
        t = time.perf_counter()
        r = s_host.forward(e_in, source=dict(src), monitors=mons)
        fom = (r.metadata["monitors"][0]["dft"].abs() ** 2).sum()
        fom.backward()
        g_el = max_over_ranks(time.perf_counter() - t, ws, dev)
        grad_e2e = {"value": ws * cells * T_SOLVE / g_el / 1e9, "unit": UNIT, "wall_s": g_el,
                    "h2d_bytes_per_step": e_in.numel() * e_in.element_size(),
                    "d2h_bytes_per_step": e_in.grad.numel() * e_in.grad.element_size() + 8,
                    "step": f"FOM = sum |DFT Ey|^2 and dFOM/deps of a {T_SOLVE}-step solve "
                            "(forward with checkpoints, replay, reverse sweep), "
                            "FDTDSolver3D(device='cpu', backward='time_reversal'), "
                            "after one untimed call"}
        if fp64_check is not None:
            g32 = e_in.grad.to(dev, torch.float64)
            fom32 = float(fom.detach())
            del r, fom, e_in
            torch.cuda.empty_cache()
            s64 = dn.FDTDSolver3D(grid_shape=SHAPE, dl=DL, wavelength_nm=1550.0,
                                  pml_layers=PML, n_steps=T_SOLVE, courant=COURANT, device=dev,
                                  dtype=torch.float64, backward="time_reversal")
            e64 = eps.to(dev).requires_grad_(True)
            r64 = s64.forward(e64, source=dict(src), monitors=mons)
            fom64 = (r64.metadata["monitors"][0]["dft"].abs() ** 2).sum()
            fom64.backward()
            fp64_check["fom_rel"] = abs(fom32 / float(fom64) - 1.0)
            fp64_check["gradient_rel_l2"] = rel_l2_dev(g32, e64.grad)
            fp64_check["what"] += "; FOM and dFOM/deps of the gradient_e2e solve likewise"
            del r64, fom64, e64, g32
        else:
            del r, fom, e_in
        torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v, _, desc, threads = oracle_sample(20, 2, preroll + Wm)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K,
                "warmup": Wm, "ms_per_step": el_max / K * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": config_dict({"timed_steps": [preroll + Wm, preroll + Wm + K]}),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic,
                             "peak_source": f"hbm_gbs of {peak_kind}",
                             "algorithmic_bytes_per_launch": BYTES_PER_CELL_STEP * cells,
                             "kernel": f"{fwd_kernel_name()} (one launch per time step)"},
                "cpu_baseline": cpu, "e2e": e2e, "adjoint": adjoint, "gradient_e2e": grad_e2e,
                "fp64_check": fp64_check,
                "clocks": cs.summary("untimed pre-roll + timed steps of the same solve"),
                "gpu_launches": K}
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# secondary workload: 64 ragged 2-D instances, forward + adjoint, one
# persistent launch each (not the default bench line)
# ---------------------------------------------------------------------------
BATCH_SIDES = (128, 192, 256, 384, 512, 768, 1024)


def batch2d_workload(n_inst=64, seed=7, tscale=1.0):
    from diffnano_b200.solvers.batch2d import BatchInstance
    from diffnano_b200.workloads import blob_eps_2d, gaussian_pulse_for_band

    g = torch.Generator().manual_seed(seed)
    sides = [BATCH_SIDES[int(i)] for i in torch.randint(0, len(BATCH_SIDES), (n_inst,), generator=g)]
    wls = torch.linspace(1450.0, 1650.0, 8).tolist()
    specs, eps = [], []
    for b, side in enumerate(sides):
        T = max(16, int(round(tscale * (1500 + (side - 128) * 4500 / 896))))
        wl = wls[b % 8]
        src = gaussian_pulse_for_band(wl, 200.0)
        src.update(row=30)
        specs.append(BatchInstance(grid_shape=(side, side), n_steps=T, dl=20.0, wavelength_nm=wl,
                                   pml_layers=20, courant=0.5, source=src,
                                   monitor={"row": side - 30, "wavelengths_nm": [wl]}))
        eps.append(blob_eps_2d(side, min(128, side - 64), seed=b // 3, variant=(b % 3) - 1))
    return specs, eps


# FP32 TMz bytes per cell-step: forward reads Ez, Hx, Hy, dt/eps and writes the
# three fields (28); a reverse step, as the 3-D adjoint is counted, is forward
# recompute 28 + adjoint update 28 + dL/deps read-modify-write 8 = 64, and moves
# 16 more (the curl record written and read back, 4 + 4; the FP64 gradient's
# extra 8)
B2D_FWD_BYTES, B2D_BWD_BYTES, B2D_BWD_MOVED = 28, 64, 80


def batch_bandwidth(cells_steps: float, f_s: float, b_s: float) -> dict:
    peak, kind = measured_peak_hbm()
    fwd = B2D_FWD_BYTES * cells_steps / f_s / 1e9
    bwd = B2D_BWD_BYTES * cells_steps / b_s / 1e9
    return {"forward_GBs": fwd, "forward_frac": fwd / peak,
            "backward_algorithmic_bytes_per_cell_step": B2D_BWD_BYTES,
            "backward_GBs": bwd, "backward_frac": bwd / peak,
            "backward_moved_GBs": B2D_BWD_MOVED * cells_steps / b_s / 1e9,
            "peak": peak, "peak_source": f"hbm_gbs of {kind}"}


def run_batch2d(args):
    from diffnano_b200.shard import rank_share, sum_over_ranks
    from diffnano_b200.solvers.batch2d import FDTDBatch2D

    ws, rank, local = dist_setup()
    dev = torch.device("cuda", local)
    specs, eps = batch2d_workload(args.batch2d_n, tscale=args.batch2d_tscale)
    if ws > 1:  # independent instances: each rank takes a cost-balanced share
        mine = rank_share([s.grid_shape[0] * s.grid_shape[1] * s.n_steps for s in specs], ws,
                          rank)
        specs, eps = [specs[i] for i in mine], [eps[i] for i in mine]
    cells_steps = sum(s.grid_shape[0] * s.grid_shape[1] * s.n_steps for s in specs)
    batch = FDTDBatch2D(specs, "TM", torch.float32, dev)
    e_dev = [e.to(dev).requires_grad_(True) for e in eps]
    fields, dfts = batch.forward(e_dev)  # warm-up (also autotunes the tile height)
    sum((d.abs() ** 2).sum() for d in dfts).backward()
    torch.cuda.synchronize(dev)
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e_dev = [e.to(dev).requires_grad_(True) for e in eps]
    barrier(ws)
    torch.cuda.synchronize(dev)
    e0.record()
    fields, dfts = batch.forward(e_dev)
    e1.record()
    sum((d.abs() ** 2).sum() for d in dfts).backward()
    e2.record()
    torch.cuda.synchronize(dev)
    f_s, b_s = e0.elapsed_time(e1) / 1e3, e1.elapsed_time(e2) / 1e3
    f_s, b_s = max_over_ranks(f_s, ws, dev), max_over_ranks(b_s, ws, dev)
    # the same forward + gradient as one CUDA-graph replay (FOM = sum |DFT|^2)
    e_in = [e.to(dev) for e in eps]
    batch.fom_gradient_graphed(e_in)  # records the graph
    torch.cuda.synchronize(dev)
    barrier(ws)
    e0.record()
    batch.fom_gradient_graphed(e_in)
    e1.record()
    torch.cuda.synchronize(dev)
    g_s = max_over_ranks(e0.elapsed_time(e1) / 1e3, ws, dev)
    fp64_check = None
    if not args.no_fp64_check:
        # the same batch through the FP64 kernels, untimed: fields, DFTs, gradients
        g32 = [e.grad.detach().double() for e in e_dev]
        f32 = [f.detach().double() for f in fields]
        d32 = [d.detach() for d in dfts]
        del fields, dfts, e_dev
        b64 = FDTDBatch2D(specs, "TM", torch.float64, dev)
        e64 = [e.to(dev).requires_grad_(True) for e in eps]
        f64, d64 = b64.forward(e64)
        sum((d.abs() ** 2).sum() for d in d64).backward()

        def agg(a, b):
            num = sum(float(torch.linalg.vector_norm(
                torch.view_as_real(x.to(torch.complex128)) - torch.view_as_real(y.to(torch.complex128))) ** 2)
                if x.is_complex() else float(torch.linalg.vector_norm(x.double() - y.double()) ** 2)
                for x, y in zip(a, b))
            den = sum(float(torch.linalg.vector_norm(
                torch.view_as_real(y.to(torch.complex128)) if y.is_complex() else y.double()) ** 2)
                for y in b)
            return math.sqrt(num / den)

        fp64_check = {"field_rel_l2": agg(f32, f64), "dft_rel_l2": agg(d32, d64),
                      "gradient_rel_l2": agg(g32, [e.grad.double() for e in e64]),
                      "what": "every instance's FP32 field, DFT and dFOM/deps vs the same batch "
                              "on the FP64 kernels; relative L2 over the whole batch"}
        del b64, e64, f64, d64
        torch.cuda.empty_cache()
    cells_steps = int(sum_over_ranks(float(cells_steps), ws, dev))
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
        if rank != 0:
            return 0
    line = {"metric": METRIC, "value": cells_steps / f_s / 1e9, "unit": UNIT, "n_gpus": ws,
            "steps": 1, "warmup": 1, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"batched_2d_tm_{len(specs)}_instances"
                                   + ("" if args.batch2d_tscale == 1.0
                                      else f"_steps_x{args.batch2d_tscale:g}"),
                       "instances": args.batch2d_n,
                       "parallelism": f"instances split over {ws} GPU(s) by cost",
                       "sides": sorted({s.grid_shape[0] for s in specs}),
                       "cell_steps": cells_steps, "tile_rows": batch.tile_rows,
                       "checkpoint_interval": batch.K},
            "forward_s": f_s, "backward_s": b_s,
            "backward_gcells": cells_steps / b_s / 1e9,
            "bandwidth": batch_bandwidth(cells_steps, f_s, b_s),
            "graphed_forward_backward_s": g_s,
            "graphed_what": "FDTDBatch2D.fom_gradient_graphed: eps upload, forward, adjoint "
                            "seeding, backward and dFOM/deps replayed as one CUDA graph "
                            "(includes the watchdog scan and status read after the replay)",
            "fp64_check": fp64_check,
            "kernels": "k_batch2d_fwd / k_batch2d_bwd (one persistent launch each)"}
    print(json.dumps(line), flush=True)
    return 0


def measured_peak_bf16():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return float(d["bf16_tflops"]), float(d["bf16_tflops_sustained"]), "measured"
    except Exception:
        return 1590.0, 1400.0, "fallback"


def run_fno(args):
    """Learned surrogate: FDTD-labelled data, BF16 tensor-core training, held-out error."""
    from diffnano_b200.surrogate.data import FDTDLabeler, TMzSetup, cell_steps, make_dataset
    from diffnano_b200.surrogate.surrogate import FNOSurrogate

    dev = torch.device("cuda", 0)
    setup = TMzSetup()
    lab = FDTDLabeler(setup, chunk=2048, device=dev)
    n_train, n_test, epochs = args.fno_samples, args.fno_test, args.fno_epochs
    make_dataset(64, 999, lab)  # warm-up: builds the solver, first launch
    torch.cuda.synchronize(dev)
    lab = FDTDLabeler(setup, chunk=2048, device=dev)
    t0 = time.perf_counter()
    designs, labels = make_dataset(n_train, 1, lab)
    torch.cuda.synchronize(dev)
    label_s = time.perf_counter() - t0
    test_d, test_l = make_dataset(n_test, 10_000, lab)
    sur = FNOSurrogate(lab, batch_size=256, lr=1e-3, device=dev, seed=0)
    with ClockSampler(0) as clocks:
        hist = sur.train_surrogate(n_epochs=epochs, designs=designs, labels=labels)
    clk = clocks.summary()
    acc = sur.accuracy(designs=test_d, labels=test_l)
    steps = int(sur.timings["train_steps"])
    flops = sur.net.gemm_flops(256) * steps
    train_s = sur.timings["train_s"]
    # inference throughput (prescreening rate), batch 256
    x = test_d[:256]
    sur.predict(x)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(10):
        sur.predict(x)
    e1.record()
    torch.cuda.synchronize(dev)
    infer_s = e0.elapsed_time(e1) / 1e3 / 10
    peak, peak_sus, kind = measured_peak_bf16()
    tflops = flops / train_s / 1e12
    line = {"metric": "FNO surrogate training throughput", "value": n_train * epochs / train_s,
            "unit": "samples/s", "n_gpus": 1, "steps": steps, "warmup": 0,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16",
            "data": "synthetic (seeded blob designs labelled by the batched FDTD)",
            "config": {"workload": "fno_4layer_w64_m16_128x128_b256", "train_designs": n_train,
                       "test_designs": n_test, "epochs": epochs, "batch": 256, "lr": 1e-3,
                       "labels": "DFT Ez, 128-point monitor line, 1500/1550/1600 nm, "
                                 "256x256 TMz FDTD 2000 steps"},
            "label_s": label_s, "label_gcells": cell_steps(n_train, setup) / label_s / 1e9,
            "train_s": train_s, "final_train_loss": hist[-1], "first_epoch_loss": hist[0],
            "heldout": acc,
            "gain_vs_no_network": acc["mean_predictor_rel_l2"] / acc["mean_rel_l2"],
            "roofline": {"bound": "tensor", "achieved": tflops, "peak": peak_sus,
                         "unit": "TFLOP/s", "frac": tflops / peak_sus,
                         "peak_kind": f"{kind} sustained bf16"},
            "infer_designs_per_s": 256 / infer_s, "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def run_design(args):
    """3-D inverse design: plain FDTD Adam loop vs surrogate-assisted loop, time to FOM."""
    from diffnano_b200.design.loop import SurrogateAssistedLoop, SurrogateConfig, plain_loop
    from diffnano_b200.design.metalens import Metalens3D, MetalensSetup

    dev = torch.device("cuda", 0)
    setup = MetalensSetup() if args.design_scale == 1 else MetalensSetup().scaled(args.design_scale)
    rho0 = torch.full(setup.design_shape, 0.5, device=dev)
    warm = Metalens3D(setup, dev)
    warm.evaluate(rho0, 1.0, grad=True)  # first launches, allocations
    del warm
    torch.cuda.synchronize(dev)
    prob = Metalens3D(setup, dev)
    with ClockSampler(0) as clocks:
        plain = plain_loop(prob, rho0, iters=args.design_iters, lr=0.02, beta=(1.0, 32.0))
    target = plain["final_fom"]
    prob2 = Metalens3D(setup, dev)
    from diffnano_b200.surrogate.fno import FNOConfig
    dz, dx = setup.design_shape
    cfg = SurrogateConfig(max_verify=args.design_max_verify, model=args.design_model,
                          fno=FNOConfig(H=dz, W=dx, modes=min(16, dz // 2 - 1),
                                        eps_lo=setup.eps_lo, eps_hi=setup.eps_hi))
    loop = SurrogateAssistedLoop(prob2, cfg)
    res = loop.run(rho0, target=target, beta=(1.0, 32.0))
    plain_s = plain["wall_s"]
    t_sur = res["time_to_target_s"]
    hist = [{"n": r.verification, "t": round(r.wall_s, 2), "fom": r.fom / plain["fom0"],
             "beta": round(r.beta, 2), "kind": r.kind} for r in res["history"]]

    def first_reach(records, thr):
        for r in records:
            if r.fom >= thr:
                return r.wall_s
        return None

    # wall time of each loop to its first FDTD-verified FOM at a fraction of
    # the plain loop's final FOM (the metric itself is the 0.99 entry)
    fractions = {}
    for f in (0.5, 0.75, 0.9, 0.95, 0.97, 0.99):
        tp = first_reach(plain["history"], f * target)
        ta = first_reach(res["history"], f * target)
        fractions[str(f)] = {"plain_s": tp, "assisted_s": ta,
                             "speedup": (tp / ta) if tp and ta else None}
    line = {"metric": "time-to-FOM speed-up, surrogate-assisted vs plain 3-D inverse design",
            "value": (plain_s / t_sur) if t_sur else None, "unit": "x", "n_gpus": 1,
            "steps": args.design_iters, "warmup": 1, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (uniform start density, seeded proxy designs)",
            "config": {"workload": "metalens3d_384x384x192_dx25_cpml12_T3000",
                       "grid_zyx": list(setup.shape), "design_zx": list(setup.design_shape),
                       "parameterisation": "rho(z,x) extruded along y, filter r=4, tanh "
                                           "projection, beta 1->32",
                       "fom": "|DFT Ey(1550 nm)|^2 at the focal point",
                       "plain": f"{args.design_iters} Adam iterations, FDTD forward+adjoint each",
                       "assisted": "model (mapped to the 3-D focal field by a fitted output "
                                   "map) gives the warm start (beta ramped to "
                                   f"{cfg.tr_beta_frac} of its end value) and proposes "
                                   f"trust-region steps (the first {cfg.tr_beta_steps} finish "
                                   f"the beta ramp); it checks the FNO's top {cfg.n_check}; the "
                                   "3-D FDTD verifies the best and judges every step",
                       "surrogate": f"FNO trained on {cfg.n_train} batched-FDTD labels of the "
                                    f"2-D cross-section prescreens {cfg.n_candidates} candidates "
                                    f"per verification; the {cfg.model} model "
                                    f"({cfg.coarse_factor}x coarser 3-D cells)"
                                    if cfg.model == "coarse3d" else
                                    f"FNO trained on {cfg.n_train} batched-FDTD labels of the "
                                    f"2-D cross-section prescreens {cfg.n_candidates} candidates "
                                    f"per verification; the cross-section model"},
            "plain": {"history": [{"n": r.verification, "t": round(r.wall_s, 2),
                                   "fom": r.fom / plain["fom0"], "beta": round(r.beta, 2)}
                                  for r in plain["history"]],
                      "wall_s": plain_s, "final_fom": target / plain["fom0"],
                      "best_fom": plain["best_fom"] / plain["fom0"],
                      "s_per_iteration": plain_s / args.design_iters,
                      "gcells": setup.cell_steps() * args.design_iters / plain_s / 1e9},
            "time_to_fraction_of_plain_fom": fractions,
            "assisted": {"wall_s": res["wall_s"], "time_to_target_s": t_sur,
                         "final_fom": res["final_fom"] / plain["fom0"],
                         "best_fom_at_final_beta": (res["best_fom"] / plain["fom0"])
                         if res["best_fom"] else None,
                         "fdtd_verifications": res["verifications"],
                         "timings": res["timings"], "proxy_heldout_rel_l2": loop.proxy_error(),
                         "model": res["model"], "output_map": res["map"],
                         "network_map": res["net_map"], "candidates": res["candidates"],
                         "history": hist},
            "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)
    return 0


def run_fdtd2d(args):
    """Config 0: the 256^2 TMz solve (2000 steps) through FDTDSolver2D, and 1024^2."""
    from diffnano_b200.solvers import FDTDSolver2D
    from diffnano_b200.surrogate.data import TMzSetup, blob_designs, design_eps

    dev = torch.device("cuda", 0)
    st = TMzSetup()
    mask, _ = blob_designs(1, 0, (3.0, 3.0))
    eps = torch.full((st.side, st.side), 2.085, dtype=torch.float64)
    o = st.offset
    eps[o:o + st.design, o:o + st.design] = design_eps(mask[0]).to(torch.float64)
    src = st.instance().source
    mon = [{"component": "Ez", "row": st.mon_row, "wavelengths_nm": list(st.wavelengths_nm)}]
    out = {}
    for side, T, key in ((st.side, st.n_steps, "cfg0"), (1024, 1000, "1024")):
        e = eps if side == st.side else torch.nn.functional.pad(eps, ((1024 - 256) // 2,) * 4,
                                                                value=2.085)
        solver = FDTDSolver2D(grid_shape=(side, side), dl=st.dl, wavelength_nm=st.center_nm,
                              pml_layers=st.pml, n_steps=T, courant=st.courant, device=dev,
                              dtype=torch.float32, monitors=mon)
        ed = e.to(dev)
        # warm-up: at least --warmup solves and half a second of solving, so that
        # the SM clock has left its idle state before the timed solves (a 256^2
        # solve is 8 ms: 20 of them were not always enough)
        n_warm, t_w = 0, time.perf_counter()
        while n_warm < args.warmup or time.perf_counter() - t_w < 0.5:
            solver.forward(ed, source=dict(src))
            n_warm += 1
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 25 if side == st.side else 5
        e0.record()
        for _ in range(reps):
            r = solver.forward(ed, source=dict(src))
        e1.record()
        torch.cuda.synchronize(dev)
        s_solve = e0.elapsed_time(e1) / 1e3 / reps
        # gradient-free solves that fit one thread-block cluster run as one
        # launch per solve; the others launch the step kernel once per step
        batch = next((v for v in solver.__dict__.get("_cluster_cache", {}).values()
                      if v is not None), None)
        cluster = batch is not None
        kernel = "k_fdtd2d_step"
        if cluster:
            from diffnano_b200 import _lib

            db = batch._cluster[0] & _lib.DN_CLUSTER_DOUBLE_BUFFERED
            kernel = "k_batch2d_cluster_db" if db else "k_batch2d_cluster"
        out[key] = {"grid": side, "steps": T, "s_per_solve": s_solve,
                    "gcells": side * side * T / s_solve / 1e9,
                    "gbs": 28 * side * side * T / s_solve / 1e9,
                    "kernel": kernel, "warmup_solves": n_warm, "timed_solves": reps,
                    "launches_per_solve": 1 if cluster else T}
        if not args.no_fp64_check:
            s64 = FDTDSolver2D(grid_shape=(side, side), dl=st.dl, wavelength_nm=st.center_nm,
                               pml_layers=st.pml, n_steps=T, courant=st.courant, device=dev,
                               dtype=torch.float64, monitors=mon)
            r64 = s64.forward(ed, source=dict(src))
            out[key]["fp64_check"] = {
                "field_rel_l2": rel_l2_dev(r.field, r64.field),
                "dft_rel_l2": rel_l2_dev(r.metadata["monitors"][0]["dft"],
                                         r64.metadata["monitors"][0]["dft"]),
                "what": "FP32 result of the timed solve vs the same solve on the FP64 kernels "
                        "(Ez field, Ez line DFT), relative L2"}
        if key == "cfg0":
            host = FDTDSolver2D(grid_shape=(side, side), dl=st.dl, wavelength_nm=st.center_nm,
                                pml_layers=st.pml, n_steps=T, courant=st.courant, device="cpu",
                                dtype=torch.float32, monitors=mon)
            ep = e.to(torch.float32).pin_memory()
            host.forward(ep, source=dict(src))
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            for _ in range(reps):
                rh = host.forward(ep, source=dict(src))
            e2e_s = (time.perf_counter() - t0) / reps
            out["e2e"] = {"value": side * side * T / e2e_s / 1e9, "unit": UNIT,
                          "h2d_bytes_per_step": 4 * side * side,
                          "d2h_bytes_per_step": 4 * side * side + 16 * 3 * side,
                          "step": "FDTDSolver2D(device='cpu').forward of the 2000-step solve"}
            del rh
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, ROOT)
        from oracle import fdtd_ref

        torch.set_num_threads(os.cpu_count() or 1)
        dt = st.courant * st.dl / math.sqrt(2.0)
        t0 = time.perf_counter()
        fdtd_ref.run_2d(eps, dl=st.dl, dt=dt, omega=2 * math.pi / st.center_nm,
                        pml_layers=st.pml, n_steps=st.n_steps, source=dict(src),
                        monitors=[{"component": "Ez", "box": ((st.mon_row, st.mon_row + 1),
                                                                (0, st.side)),
                                   "wavelengths_nm": list(st.wavelengths_nm)}])
        cpu_s = time.perf_counter() - t0
        cpu = {"value": st.side * st.side * st.n_steps / cpu_s / 1e9, "unit": UNIT,
               "cores": torch.get_num_threads(), "kind": "port",
               "sample": "the full 256^2 x 2000-step solve, FP64 torch-CPU restatement of "
                         "fdtd2d.py:_time_step_tm (oracle/fdtd_ref.py)"}
    peak, _ = measured_peak_hbm()
    c0 = out["cfg0"]
    c0_launches = c0["timed_solves"] * c0["launches_per_solve"]
    line = {"metric": METRIC, "value": c0["gcells"], "unit": UNIT, "n_gpus": 1,
            "steps": c0["steps"], "warmup": c0["warmup_solves"],
            "ms_per_step": c0["s_per_solve"] / c0["steps"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "2d_tmz_256x256_cpml20_2000steps (state L2-resident)",
                       "source": "Gaussian line source row 30, 1550 nm, 200 nm band",
                       "monitor": "Ez row 226 at 1500/1550/1600 nm"},
            "grid_1024": out["1024"],
            "roofline": {"bound": "hbm", "achieved": out["1024"]["gbs"], "peak": peak,
                         "unit": "GB/s", "frac": out["1024"]["gbs"] / peak,
                         "note": "1024^2 grid (28 B/cell-step); 256^2 is L2-resident"},
            "e2e": out["e2e"], "cpu_baseline": cpu,
            "fp64_check": c0.get("fp64_check"),
            "gpu_launches": c0_launches,
            "kernels": f"{c0['kernel']} ({c0['launches_per_solve']} launch(es) per solve, {c0['timed_solves']} solves "
                       f"timed); grid_1024: {out['1024']['kernel']}"}
    print(json.dumps(line), flush=True)
    return 0


def run_fdtd3d_phases(args):
    """Diagnostics of the 3-D workload (no bench line): per-step time over 500-step
    segments of a 4000-step solve, continuing vs restarting each segment from the
    zero state, and the phases of one host-in / host-out FDTDSolver3D solve."""
    import diffnano_b200 as dn
    from diffnano_b200.solvers._adjoint import run_forward

    dev = torch.device("cuda", 0)
    eps, src, mons = workload()
    solver = dn.FDTDSolver3D(grid_shape=SHAPE, dl=DL, wavelength_nm=1550.0, pml_layers=PML,
                             n_steps=T_SOLVE, courant=COURANT, device=dev, dtype=torch.float32)
    eng = solver._make_engine(T_SOLVE, dict(src), mons)
    eng.set_eps(eps.to(dev))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    seg = 500
    out = {"segment_steps": seg}
    for mode in ("continue", "restart_each"):
        eng.reset()
        t, times = 0, []
        for _ in range(T_SOLVE // seg):
            if mode == "restart_each":
                eng.reset()
                t = 0
            torch.cuda.synchronize(dev)
            e0.record()
            eng.run(t, seg)
            e1.record()
            torch.cuda.synchronize(dev)
            times.append(round(e0.elapsed_time(e1) / seg, 4))
            t += seg
        out[f"ms_per_step_{mode}"] = times
    eng.check_status()
    del eng
    torch.cuda.empty_cache()

    def tick():
        torch.cuda.synchronize(dev)
        return time.perf_counter()

    host = dn.FDTDSolver3D(grid_shape=SHAPE, dl=DL, wavelength_nm=1550.0, pml_layers=PML,
                           n_steps=T_SOLVE, courant=COURANT, device="cpu", dtype=torch.float32)
    ep = eps.to(torch.float32).pin_memory()
    host.forward(ep, source=dict(src), monitors=mons)  # warm-up
    t0 = tick()
    host.forward(ep, source=dict(src), monitors=mons)
    out["host_forward_s"] = round(tick() - t0, 4)
    t0 = tick()
    eng = host._make_engine(T_SOLVE, dict(src), mons)
    out["engine_setup_s"] = round(tick() - t0, 4)
    t0 = tick()
    field, _ = run_forward(host, eng, host._prep_eps(ep), ("Ez", "Ex", "Ey"))
    out["solve_s"] = round(tick() - t0, 4)
    t0 = tick()
    field.to("cpu")
    out["field_to_pageable_host_s"] = round(tick() - t0, 4)
    pinned = torch.empty(field.shape, dtype=field.dtype, pin_memory=True)
    t0 = tick()
    pinned.copy_(field, non_blocking=True)
    out["field_to_pinned_host_s"] = round(tick() - t0, 4)
    out["field_bytes"] = field.numel() * field.element_size()
    del eng, field, pinned
    torch.cuda.empty_cache()

    # the gradient call of the bench line, split into forward and backward
    gs = dn.FDTDSolver3D(grid_shape=SHAPE, dl=DL, wavelength_nm=1550.0, pml_layers=PML,
                         n_steps=T_SOLVE, courant=COURANT, device="cpu", dtype=torch.float32,
                         backward="time_reversal")
    for rep in range(2):
        e_in = eps.to(torch.float32).pin_memory().requires_grad_(True)
        t0 = tick()
        r = gs.forward(e_in, source=dict(src), monitors=mons)
        fom = (r.metadata["monitors"][0]["dft"].abs() ** 2).sum()
        t1 = tick()
        fom.backward()
        t2 = tick()
        out[f"grad_forward_s_{rep}"] = round(t1 - t0, 4)
        out[f"grad_backward_s_{rep}"] = round(t2 - t1, 4)
        del r, fom, e_in
    print(json.dumps(out), flush=True)
    return 0


def run_gemm(args):
    """tcgen05 BF16 GEMM alone: a square GEMM and the operator's transform shape."""
    from diffnano_b200.surrogate.gemm import OutMap, gemm, kmajor

    dev = torch.device("cuda", 0)
    n = args.gemm_n
    a = torch.randn(n, n, device=dev).to(torch.bfloat16)
    b = torch.randn(n, n, device=dev).to(torch.bfloat16)
    o = torch.empty(n, n, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize(dev)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / reps

    ms = timed(lambda: gemm(n, n, [(kmajor(a, n, n), kmajor(b, n, n))], o, OutMap.rowmajor(n),
                            pair=args.gemm_pair), args.steps)
    ref = a[:128].float() @ b.float().T
    err = float((o[:128] - ref).norm() / ref.norm())
    mt = torch.matmul(a, b.T)
    ms_ref = timed(lambda: torch.matmul(a, b.T, out=mt), args.steps)
    peak, peak_sus, kind = measured_peak_bf16()
    tf = 2 * n ** 3 / ms / 1e9
    line = {"metric": "BF16 GEMM TFLOP/s (tcgen05, FP32 accumulate)", "value": tf,
            "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16",
            "data": "synthetic",
            "config": {"workload": f"gemm_{n}x{n}x{n}_bf16",
                       "tiles": {0: "one-CTA 128x256", 1: "one-CTA 128x256",
                                 2: "two-CTA 256x256"}[args.gemm_pair]},
            "rel_err_vs_fp32": err, "torch_matmul_tflops": 2 * n ** 3 / ms_ref / 1e9,
            "roofline": {"bound": "tensor", "achieved": tf, "peak": peak, "unit": "TFLOP/s",
                         "frac": tf / peak, "peak_kind": f"{kind} burst bf16"}}
    print(json.dumps(line), flush=True)
    return 0


def run_fno_step(args):
    """Operator training steps (forward, MSE, backward, Adam) on synthetic inputs."""
    from diffnano_b200.surrogate.fno import FNO2d, FNOConfig

    dev = torch.device("cuda", 0)
    B = args.fno_batch
    net = FNO2d(FNOConfig(), dev, seed=0)
    g = torch.Generator(device=dev).manual_seed(0)
    eps = 2.085 + 10.0 * torch.rand(B, 128, 128, device=dev, generator=g)
    tgt = 0.1 * torch.randn(B, 128, 6, device=dev, generator=g)

    def step():
        net.forward(eps)
        net.loss(tgt)
        net.ps.g.zero_()
        net.backward(B=B)
        net.adam_step()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    net.check_status()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / args.steps
    peak, peak_sus, kind = measured_peak_bf16()
    tf = net.gemm_flops(B) / ms / 1e9
    line = {"metric": "FNO training step throughput", "value": B / ms * 1e3,
            "unit": "samples/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16", "data": "synthetic",
            "config": {"workload": f"fno_4layer_w64_m16_128x128_b{B}"},
            "roofline": {"bound": "tensor", "achieved": tf, "peak": peak_sus, "unit": "TFLOP/s",
                         "frac": tf / peak_sus, "peak_kind": f"{kind} sustained bf16",
                         "flops": "useful GEMM FLOPs of forward + backward"}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--adjoint-steps", type=int, default=256)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-grad-e2e", action="store_true")
    ap.add_argument("--no-fp64-check", action="store_true",
                    help="skip the untimed FP64 cross-run of the solve and its gradient")
    ap.add_argument("--workload", choices=["fdtd3d", "fdtd2d", "batch2d", "fno", "design",
                                           "gemm", "fno-step", "fdtd3d-phases"],
                    default="fdtd3d",
                    help="fdtd3d: the benchmark (3-D 256^3); batch2d: 64 ragged 2-D instances; "
                         "fno: surrogate data generation + training; design: 3-D inverse "
                         "design, plain vs surrogate-assisted")
    ap.add_argument("--gemm-n", type=int, default=8192)
    ap.add_argument("--gemm-pair", type=int, default=0, choices=[0, 1, 2],
                    help="GEMM tiles: 0 or 1 one-CTA, 2 two-CTA pairs")
    ap.add_argument("--batch2d-n", type=int, default=64,
                    help="instances of the batched 2-D workload (64 is the workload)")
    ap.add_argument("--batch2d-tscale", type=float, default=1.0,
                    help="scale the step counts (1 is the workload; smaller for profiling)")
    ap.add_argument("--fno-batch", type=int, default=256)
    ap.add_argument("--design-iters", type=int, default=100)
    ap.add_argument("--design-max-verify", type=int, default=60)
    ap.add_argument("--design-model", choices=["coarse3d", "cross-section"], default="coarse3d",
                    help="proposing model of the assisted design loop")
    ap.add_argument("--design-scale", type=int, default=1,
                    help="shrink the design workload's grid by this factor (tests)")
    ap.add_argument("--fno-samples", type=int, default=20000)
    ap.add_argument("--fno-test", type=int, default=1024)
    ap.add_argument("--fno-epochs", type=int, default=50)
    ap.add_argument("--grid", type=int, default=256,
                    help="cubic grid side (256 is the benchmark; smaller sides are for profiling)")
    args = ap.parse_args()
    global SHAPE
    SHAPE = (args.grid,) * 3
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch2d":
        return run_batch2d(args)
    if args.workload == "fno":
        return run_fno(args)
    if args.workload == "design":
        return run_design(args)
    if args.workload == "fdtd3d-phases":
        return run_fdtd3d_phases(args)
    if args.workload == "gemm":
        return run_gemm(args)
    if args.workload == "fdtd2d":
        return run_fdtd2d(args)
    if args.workload == "fno-step":
        return run_fno_step(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
