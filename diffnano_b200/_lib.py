"""ctypes binding of the C ABI in ``include/dn_fdtd.h`` (``_native/libdn_fdtd.so``).

The library is built in-tree by ``diffnano_b200/build.py``.  There is no
fallback: if the library is missing, :func:`lib` raises.
"""

from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_native", "libdn_fdtd.so")

# status codes (dn_fdtd.h)
DN_OK, DN_EINVAL, DN_ENOMEM, DN_ECUDA, DN_ETIMEOUT, DN_ENONFINITE, DN_EUNSUPPORTED = range(7)
DN_F32, DN_F64 = 0, 1
DN_EX, DN_EY, DN_EZ, DN_HX, DN_HY, DN_HZ = range(6)
DN_NONE = -1
DN_TM, DN_TE = 0, 1
DN_CLUSTER_DOUBLE_BUFFERED = 0x100  # flag in dn_batch2d_cluster_size's result
DN_AXES_REFERENCE, DN_AXES_PHYSICAL = 0, 1
DN_MAX_MONITORS = 4
DN_MAX_FREQS = 16
DN_NOALLOC_MAX_BYTES = 6 * 1024 * 1024

COMPONENTS = {"Ex": DN_EX, "Ey": DN_EY, "Ez": DN_EZ, "Hx": DN_HX, "Hy": DN_HY, "Hz": DN_HZ}

c_int32, c_int64, c_double, c_void_p = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p


class DnBox(ctypes.Structure):
    _fields_ = [("lo", c_int32 * 3), ("hi", c_int32 * 3)]


class DnGrid(ctypes.Structure):
    _fields_ = [("D", c_int32), ("H", c_int32), ("W", c_int32), ("dtype", c_int32),
                ("pitch_y", c_int64), ("pitch_z", c_int64), ("dt", c_double), ("dl", c_double),
                ("axes", c_int32), ("pol", c_int32)]


class DnCpml(ctypes.Structure):
    _fields_ = [("b", c_void_p * 3), ("c", c_void_p * 3)]


class DnSource(ctypes.Structure):
    _fields_ = [("component", c_int32), ("box", DnBox), ("wave", c_void_p), ("n_t", c_int32)]


class DnMonitor(ctypes.Structure):
    _fields_ = [("component", c_int32), ("box", DnBox), ("n_freq", c_int32),
                ("phase", c_void_p), ("acc", c_void_p), ("n_t", c_int32)]


class DnProbe(ctypes.Structure):
    _fields_ = [("component", c_int32), ("pos", c_int32 * 3), ("out", c_void_p),
                ("n_t", c_int32)]


class DnCurlRecord(ctypes.Structure):
    _fields_ = [("curl", c_void_p * 3), ("step_stride", c_int64), ("t0", c_int32),
                ("nslots", c_int32)]


class DnBatch2dInst(ctypes.Structure):
    _fields_ = [("H", c_int32), ("W", c_int32), ("pitch", c_int64), ("n_steps", c_int32),
                ("src_comp", c_int32), ("src_box", DnBox), ("wave", c_void_p),
                ("f", (c_void_p * 3) * 2), ("ce", c_void_p), ("b", c_void_p * 2),
                ("c", c_void_p * 2), ("dt", c_double), ("dl", c_double), ("mon_comp", c_int32),
                ("mon_box", DnBox), ("n_freq", c_int32), ("phase", c_void_p), ("acc", c_void_p),
                ("ckpt", c_void_p), ("curl", c_void_p), ("lam", (c_void_p * 3) * 2),
                ("grad", c_void_p), ("gmon", c_void_p)]


class DnBatch2d(ctypes.Structure):
    _fields_ = [("pol", c_int32), ("dtype", c_int32), ("n_inst", c_int32), ("K", c_int32),
                ("tile_rows", c_int32), ("max_ctas", c_int32)]


class DnGemmOperand(ctypes.Structure):
    _fields_ = [("ptr", c_void_p), ("mn_major", c_int32), ("fold", c_int32), ("rows", c_int64),
                ("k", c_int64), ("ld", c_int64), ("fold_stride", c_int64),
                ("batch_stride", c_int64)]


class DnGemm(ctypes.Structure):
    _fields_ = [("M", c_int64), ("N", c_int64), ("batch", c_int32), ("n_seg", c_int32),
                ("a", DnGemmOperand * 2), ("b", DnGemmOperand * 2), ("out", c_void_p),
                ("out_dtype", c_int32), ("accumulate", c_int32), ("c_batch_stride", c_int64),
                ("c_row_radix", c_int64), ("c_row_stride0", c_int64), ("c_row_stride1", c_int64),
                ("c_col_radix", c_int64), ("c_col_stride0", c_int64), ("c_col_stride1", c_int64),
                ("alpha", ctypes.c_float), ("act", c_int32), ("bias", c_void_p),
                ("row_scale", c_void_p), ("batch_scale", c_void_p), ("addend", c_void_p),
                ("addend_dtype", c_int32), ("aux_dtype", c_int32), ("aux", c_void_p),
                ("pre", c_void_p), ("pre_dtype", c_int32), ("block_n", c_int32),
                ("max_ctas", c_int32), ("col_scale", c_void_p), ("row_bias", c_void_p),
                ("pair", c_int32)]


class DnDensity(ctypes.Structure):
    _fields_ = [("n_layers", c_int32), ("H", c_int32), ("W", c_int32), ("kind", c_int32),
                ("radius", ctypes.c_float), ("beta", ctypes.c_float), ("eta", ctypes.c_float),
                ("eps_lo", ctypes.c_float), ("eps_hi", ctypes.c_float)]


class DnSpan(ctypes.Structure):
    _fields_ = [("ptr", c_void_p), ("dtype", c_int32), ("rows", c_int64), ("cols", c_int64),
                ("pitch", c_int64)]


DN_MAX_SPANS = 32

STRUCTS = {"dn_box": DnBox, "dn_grid": DnGrid, "dn_cpml": DnCpml, "dn_source": DnSource,
           "dn_monitor": DnMonitor, "dn_probe": DnProbe, "dn_curl_record": DnCurlRecord,
           "dn_batch2d_inst": DnBatch2dInst, "dn_batch2d": DnBatch2d,
           "dn_gemm_operand": DnGemmOperand, "dn_gemm": DnGemm,
           "dn_density": DnDensity, "dn_span": DnSpan}

PTR6 = c_void_p * 6
_P6 = ctypes.POINTER(c_void_p)  # a PTR6 instance (or None) is passed here

# name -> (restype, argtypes); every symbol include/dn_fdtd.h declares
SIGNATURES = {
    "dn_strerror": (ctypes.c_char_p, [c_int32]),
    "dn_version": (c_int32, []),
    "dn_last_cuda_error": (c_int32, []),
    "dn_fdtd2d_run": (c_int32, [ctypes.POINTER(DnGrid), _P6, _P6, c_void_p,
                                ctypes.POINTER(DnCpml), ctypes.POINTER(DnSource),
                                ctypes.POINTER(DnMonitor), c_int32, ctypes.POINTER(DnProbe),
                                ctypes.POINTER(DnCurlRecord), c_int32, c_int32, c_void_p,
                                c_void_p, ctypes.POINTER(c_int32)]),
    "dn_fdtd3d_run": (c_int32, [ctypes.POINTER(DnGrid), _P6, _P6, c_void_p,
                                ctypes.POINTER(DnCpml), ctypes.POINTER(DnSource),
                                ctypes.POINTER(DnMonitor), c_int32, ctypes.POINTER(DnProbe),
                                ctypes.POINTER(DnCurlRecord), c_int32, c_int32, c_void_p,
                                c_void_p, ctypes.POINTER(c_int32)]),
    "dn_fdtd2d_adjoint": (c_int32, [ctypes.POINTER(DnGrid), _P6, _P6, c_void_p,
                                    ctypes.POINTER(DnCpml), ctypes.POINTER(DnCurlRecord),
                                    c_void_p, ctypes.POINTER(DnMonitor), c_int32, c_int32,
                                    c_int32, c_void_p, c_void_p, ctypes.POINTER(c_int32)]),
    "dn_fdtd3d_adjoint": (c_int32, [ctypes.POINTER(DnGrid), _P6, _P6, c_void_p,
                                    ctypes.POINTER(DnCpml), ctypes.POINTER(DnCurlRecord),
                                    c_void_p, ctypes.POINTER(DnMonitor), c_int32, c_int32,
                                    c_int32, c_void_p, c_void_p, ctypes.POINTER(c_int32)]),
    "dn_struct_size": (c_int64, [ctypes.c_char_p]),
    "dn_batch2d_table_bytes": (c_int64, [ctypes.POINTER(DnBatch2d), ctypes.POINTER(DnBatch2dInst)]),
    "dn_batch2d_pack": (c_int32, [ctypes.POINTER(DnBatch2d), ctypes.POINTER(DnBatch2dInst),
                                  c_void_p, c_int64]),
    "dn_batch2d_forward": (c_int32, [ctypes.POINTER(DnBatch2d), c_void_p, c_void_p, c_void_p]),
    "dn_batch2d_backward": (c_int32, [ctypes.POINTER(DnBatch2d), c_void_p, c_void_p, c_void_p]),
    "dn_batch2d_cluster_size": (c_int32, [ctypes.POINTER(DnBatch2d), ctypes.POINTER(DnBatch2dInst),
                                          ctypes.POINTER(c_int64)]),
    "dn_batch2d_forward_cluster": (c_int32, [ctypes.POINTER(DnBatch2d), c_void_p, c_int32,
                                             c_int64, c_void_p]),
    "dn_batch2d_barrier_selftest": (c_int32, [c_int32, c_int32, c_int64, c_int32, c_void_p,
                                              c_void_p, c_void_p]),
    "dn_fom_abs2_scratch_bytes": (c_int64, [c_int64]),
    "dn_fom_abs2": (c_int32, [c_void_p, c_int64, c_void_p, c_void_p, c_int64, c_void_p]),
    "dn_gemm_run": (c_int32, [ctypes.POINTER(DnGemm), c_void_p, c_void_p]),
    "dn_fno_features": (c_int32, [c_void_p, c_int64, c_int32, c_int32, ctypes.c_float,
                                  ctypes.c_float, c_void_p, c_void_p]),
    "dn_fno_lift": (c_int32, [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_int32,
                              c_void_p, c_void_p]),
    "dn_fno_features_bwd": (c_int32, [c_void_p, c_int64, ctypes.c_float, ctypes.c_float,
                                      c_void_p, c_void_p]),
    "dn_fno_readout": (c_int32, [c_void_p, c_void_p, c_int64, c_int32, c_int32, c_int32,
                                 c_void_p, c_void_p]),
    "dn_fno_readout_bwd": (c_int32, [c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_int32,
                                     c_int32, c_void_p, c_void_p, c_void_p]),
    "dn_colsum_scratch_elems": (c_int64, [c_int64, c_int64]),
    "dn_colsum": (c_int32, [c_void_p, c_int32, c_int64, c_int64, c_int64, c_void_p, c_int32,
                            c_void_p, c_int64, c_void_p]),
    "dn_mse": (c_int32, [c_void_p, c_void_p, c_int64, c_int32, c_int32, ctypes.c_float,
                         c_void_p, c_void_p, c_int32, c_void_p]),
    "dn_adam": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, ctypes.c_float,
                          ctypes.c_float, ctypes.c_float, ctypes.c_float, c_int32,
                          ctypes.c_float, c_void_p, c_void_p]),
    "dn_fno_pack_modes": (c_int32, [c_void_p, c_void_p, c_int64, c_int32, c_int32, c_void_p,
                                    c_void_p]),
    "dn_fno_unpack_mode_grads": (c_int32, [c_void_p, c_int64, c_int32, c_int32, c_void_p,
                                           c_void_p, c_void_p]),
    "dn_f32_to_bf16": (c_int32, [c_void_p, c_int64, c_void_p, c_void_p]),
    "dn_fno_channel_sums": (c_int32, [c_void_p, c_int64, c_int32, c_int64, c_void_p, c_void_p,
                                      c_void_p]),
    "dn_fno_pack_pointwise": (c_int32, [c_void_p, c_void_p, c_int32, c_void_p, c_void_p,
                                        c_void_p, c_void_p]),
    "dn_fno_modes_rows": (c_int32, [c_void_p, c_void_p, c_int32, c_int64, c_int32, c_int32,
                                    c_void_p]),
    "dn_density_forward": (c_int32, [ctypes.POINTER(DnDensity), c_void_p, c_void_p, c_void_p,
                                     c_void_p, c_void_p]),
    "dn_density_backward": (c_int32, [ctypes.POINTER(DnDensity), c_void_p, c_void_p, c_void_p,
                                      c_void_p, c_void_p]),
    "dn_morph3": (c_int32, [c_void_p, c_int32, c_int32, c_int32, c_int32, c_void_p, c_void_p,
                            c_void_p]),
    "dn_morph3_backward": (c_int32, [c_void_p, c_void_p, c_int32, c_int32, c_int32, c_void_p,
                                     c_void_p]),
    "dn_check_finite": (c_int32, [ctypes.POINTER(DnSpan), c_int32, c_void_p, c_void_p]),
    "dn_fdtd2d_run_noalloc": (c_int32, [ctypes.POINTER(DnGrid), _P6, c_void_p,
                                        ctypes.POINTER(DnCpml), ctypes.POINTER(DnSource),
                                        ctypes.POINTER(DnMonitor), c_int32,
                                        ctypes.POINTER(DnProbe), c_int32, c_int32, c_void_p,
                                        c_void_p]),
}


class DNError(RuntimeError):
    """A dn_* call returned a non-OK status."""

    def __init__(self, fn: str, status: int, msg: str):
        super().__init__(f"{fn} failed: {msg} (status {status})")
        self.status = status


_lock = threading.Lock()
_lib = None


def lib() -> ctypes.CDLL:
    """Load the CUDA library (once).  Raises if it has not been built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"diffnano_b200 CUDA library not built ({LIB_PATH} missing); run "
                    "`python -c 'import __graft_entry__ as g; g.build()'` or "
                    "`python diffnano_b200/build.py`")
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _lib = L
    return _lib


def check(fn: str, status: int) -> None:
    """Raise for a non-OK status (``ValueError`` for bad arguments)."""
    if status == DN_OK:
        return
    L = lib()
    msg = L.dn_strerror(status).decode()
    if status == DN_ECUDA:
        msg += f" (cuda error {L.dn_last_cuda_error()})"
    if status == DN_EINVAL:
        raise ValueError(f"{fn}: {msg}")
    raise DNError(fn, status, msg)


def spans(t) -> list:
    """:class:`DnSpan` list covering a CUDA float32/float64 tensor.

    A contiguous tensor is cut into rows of 1024 elements (plus one short
    row for the remainder); any other tensor must have unit inner stride and
    rows at a constant stride (e.g. a view that narrows the last dimension of
    a padded field), and its rows are its last dimension."""
    torch = _torch()
    if t.dtype not in (torch.float32, torch.float64):
        raise ValueError("spans: a float32 or float64 tensor is required")
    dt = DN_F32 if t.dtype == torch.float32 else DN_F64
    n = t.numel()
    if t.is_contiguous():
        out, full = [], n // 1024
        if full:
            out.append(DnSpan(ptr=t.data_ptr(), dtype=dt, rows=full, cols=1024, pitch=1024))
        if n % 1024:
            out.append(DnSpan(ptr=t.data_ptr() + full * 1024 * t.element_size(), dtype=dt,
                              rows=1, cols=n % 1024, pitch=n % 1024))
        return out
    if t.stride(-1) != 1 or t.dim() < 2:
        raise ValueError("spans: unit inner stride is required")
    for d in range(t.dim() - 2):  # leading dimensions must fold into whole rows
        if t.stride(d) != t.stride(d + 1) * t.shape[d + 1]:
            raise ValueError("spans: leading dimensions are not a constant row stride")
    cols = t.shape[-1]
    return [DnSpan(ptr=t.data_ptr(), dtype=dt, rows=n // cols, cols=cols, pitch=t.stride(-2))]


def check_finite(tensors, status, stream) -> None:
    """Queue the non-finite watchdog (``dn_check_finite``) over CUDA tensors
    on ``stream``; a NaN or Inf sets DN_ENONFINITE in the device word
    ``status`` (read later by the caller's status check)."""
    sp = [x for t in tensors if t is not None and t.numel() > 0 for x in spans(t)]
    for i in range(0, len(sp), DN_MAX_SPANS):
        chunk = sp[i:i + DN_MAX_SPANS]
        arr = (DnSpan * len(chunk))(*chunk)
        check("dn_check_finite",
              lib().dn_check_finite(arr, len(chunk), status.data_ptr(), ctypes.c_void_p(stream)))


def _torch():
    import torch

    return torch


def box(lo, hi) -> DnBox:
    b = DnBox()
    for a in range(3):
        b.lo[a] = int(lo[a])
        b.hi[a] = int(hi[a])
    return b
