"""Cross-validation against other FDTD solvers through JSON result files.

The reference's ``ExternalCrossValidator`` (``diffnano/solvers/fdtd_benchmark.py:219-310``)
reads pre-computed results of an external solver from JSON -- ``{"field": {"shape":
[...], "data": [...]}, "gradient": {...}, <anything else>}`` -- and compares them with
its own outputs (relative L2 for fields, cosine similarity for gradients).  The same
interface here, plus :func:`save_results`, which writes this solver's outputs in that
format so that either side can be the "external" one (and so that results can be kept
as golden files).
"""
from __future__ import annotations

import json
from pathlib import Path
from typing import Any, Dict, Optional, Tuple

import torch
from torch import Tensor


def _cosine_sim(a: Tensor, b: Tensor) -> float:
    a = a.detach().to(torch.float64).reshape(-1)
    b = b.detach().to(torch.float64).reshape(-1)
    den = a.norm() * b.norm()
    return float((a @ b) / den) if float(den) > 0 else 0.0


def _tensor_entry(t: Tensor) -> Dict[str, Any]:
    if t.is_complex():
        raise ValueError("complex tensors: store real and imaginary parts separately")
    t = t.detach().to("cpu", torch.float64)
    return {"shape": list(t.shape), "data": t.reshape(-1).tolist()}


def save_results(path: str, field: Optional[Tensor] = None, gradient: Optional[Tensor] = None,
                 **meta: Any) -> None:
    """Write ``field`` / ``gradient`` (and JSON-serialisable metadata) in the
    format :meth:`ExternalCrossValidator.load_external_results` reads."""
    out: Dict[str, Any] = {}
    if field is not None:
        out["field"] = _tensor_entry(field)
    if gradient is not None:
        out["gradient"] = _tensor_entry(gradient)
    for k, v in meta.items():
        if k in ("field", "gradient"):
            raise ValueError(f"metadata key {k!r} is reserved")
        out[k] = v
    Path(path).write_text(json.dumps(out))


class ExternalCrossValidator:
    """Compare this solver's outputs with an external solver's (same methods
    and return values as the reference's class)."""

    def validate_forward(self, our_result: Tensor, external_result: Tensor,
                         rtol: float = 1e-3) -> Dict[str, Any]:
        ours = our_result.detach().to("cpu", torch.float64)
        ext = external_result.detach().to("cpu", torch.float64)
        diff = ours - ext
        rel = float(diff.norm()) / max(float(ext.norm()), 1e-30)
        return {"relative_error": rel, "max_absolute_error": float(diff.abs().max()),
                "passed": rel < rtol}

    def validate_gradient(self, our_grad: Tensor, external_grad: Tensor,
                          cosine_threshold: float = 0.99) -> Dict[str, Any]:
        ours = our_grad.detach().to("cpu", torch.float64)
        ext = external_grad.detach().to("cpu", torch.float64)
        cos = _cosine_sim(ours, ext)
        rel = float((ours - ext).norm()) / max(float(ext.norm()), 1e-30)
        return {"cosine_similarity": cos, "relative_error": rel, "passed": cos >= cosine_threshold}

    def generate_test_case(self, grid_size: Tuple[int, int, int] = (16, 16, 16),
                           source_pos: Optional[Tuple[int, int, int]] = None,
                           freq: float = 1.0) -> Dict[str, Any]:
        """The reference's seeded case: eps = 1.5 + U(0,1) from seed 42 (drawn
        from a private generator: the same numbers without touching torch's
        global seed)."""
        D, H, W = grid_size
        if source_pos is None:
            source_pos = (D // 2, H // 2, W // 2)
        g = torch.Generator().manual_seed(42)
        eps = 1.5 + 1.0 * torch.rand(D, H, W, dtype=torch.float64, generator=g)
        return {"grid_size": grid_size, "source_pos": source_pos, "freq": freq, "eps": eps,
                "source_config": {"type": "gaussian_pulse", "pos": list(source_pos),
                                  "amplitude": 1.0},
                "n_steps": 50, "dl": 20.0, "wavelength_nm": 1550.0, "courant": 0.35, "seed": 42}

    @staticmethod
    def load_external_results(path: str) -> Dict[str, Any]:
        raw = json.loads(Path(path).read_text())
        result: Dict[str, Any] = {}
        for key in ("field", "gradient"):
            if key in raw:
                entry = raw[key]
                result[key] = torch.tensor(entry["data"], dtype=torch.float64).reshape(
                    tuple(entry["shape"]))
        for k, v in raw.items():
            if k not in ("field", "gradient"):
                result[k] = v
        return result
