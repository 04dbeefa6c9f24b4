"""Shared pytest configuration: the ``gpu`` marker, golden-fixture loaders and
comparison helpers.

``-m "not gpu"`` runs the oracle-vs-golden checks, host logic and the C-ABI
load/export checks (no device needed); ``-m gpu`` runs the parity tests of
the CUDA library against the oracle and the golden fixtures.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

# Parity bar of the hot path: FP64 results within 1e-12 of the reference,
# relative to the array's max magnitude (only summation order and libm
# rounding differ).
REL_TOL = 1e-12


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def rel_err(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.abs(b).max() if b.size else 0.0
    diff = np.abs(a - b).max() if b.size else 0.0
    return float(diff / scale) if scale > 0 else float(diff)


def sparse_rel_err(A, B) -> float:
    """max |A - B| / max |B| over the union pattern."""
    D = (A - B).tocoo()
    scale = np.abs(B.data).max() if B.nnz else 1.0
    return float(np.abs(D.data).max() / scale) if D.nnz else 0.0


class Golden:
    """Lazy view of one golden .npz: ``g.mesh("B")``, ``g.state(label, key)``."""

    def __init__(self, name: str):
        self.path = GOLDEN / f"{name}.npz"
        self.z = np.load(self.path)
        self.labels = sorted({k.split("/")[0] for k in self.z.files
                              if not k.startswith("mesh/")})

    def mesh(self, key):
        return self.z[f"mesh/{key}"]

    def has(self, label, key):
        return f"{label}/{key}" in self.z.files

    def state(self, label, key):
        return self.z[f"{label}/{key}"]


@pytest.fixture(scope="session")
def small_golden():
    return Golden("small_bump")


@pytest.fixture(scope="session")
def c1_golden():
    return Golden("c1_bump")


@pytest.fixture(scope="session")
def picard_golden():
    return np.load(GOLDEN / "c1_picard.npz")


def has_cuda() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
