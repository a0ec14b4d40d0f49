"""Shared test configuration: markers, paths and golden-fixture helpers."""

from __future__ import annotations

import json
import math
import os
import sys

import numpy as np
import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running test")


def load_golden(name: str) -> dict:
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    if "source" in d:
        d["source"] = json.loads(str(d["source"]))
    return d


def cfg0_eps(mask: np.ndarray) -> torch.Tensor:
    """The 256x256 config-0 eps map rebuilt from the stored design mask."""
    m = torch.tensor(mask.astype(np.float64))
    eps = torch.full((256, 256), 2.085, dtype=torch.float64)
    eps[64:192, 64:192] = 2.085 + (12.1 - 2.085) * m
    return eps


def rel_l2(a, b) -> float:
    a, b = torch.as_tensor(a).detach().cpu(), torch.as_tensor(b).detach().cpu()
    a = (torch.view_as_real(a.to(torch.complex128)) if a.is_complex() or b.is_complex()
         else a.to(torch.float64))
    b = (torch.view_as_real(b.to(torch.complex128)) if b.is_complex() or a.dim() > b.dim()
         else b.to(torch.float64))
    return float(torch.linalg.vector_norm(a - b) / max(float(torch.linalg.vector_norm(b)), 1e-300))


DT2 = lambda courant, dl: courant * dl / math.sqrt(2.0)  # noqa: E731
DT3 = lambda courant, dl: courant * dl / math.sqrt(3.0)  # noqa: E731
OMEGA = 2 * math.pi / 1550.0


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device for GPU tests (fails loudly when there is none)."""
    assert torch.cuda.is_available(), "GPU test collected on a machine without CUDA"
    return torch.device("cuda", 0)
