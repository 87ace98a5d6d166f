"""Shared fixtures and markers of the test suite.

``-m "not gpu"``: the CPU oracle against the reference's golden vectors, the host
logic of the package and the C-ABI library's exports (no GPU calls).
``-m gpu``: parity of the CUDA library against the oracle, through the C ABI.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


def golden(name: str):
    """The fixture file ``tests/golden/<name>.npz`` as a dict of arrays."""
    with np.load(GOLDEN / f"{name}.npz") as data:
        return {k: data[k] for k in data.files}


def relative(a, b) -> float:
    """The normwise relative difference max|a - b| / max|b| of the reference's tests."""
    a, b = np.asarray(a), np.asarray(b)
    scale = np.max(np.abs(b)) if b.size else 0.0
    return float(np.max(np.abs(a - b)) / scale) if scale else float(np.max(np.abs(a - b), initial=0.0))


@pytest.fixture(scope="session")
def oracle():
    from oracle import flat_tree_oracle

    flat_tree_oracle.lib()
    return flat_tree_oracle
