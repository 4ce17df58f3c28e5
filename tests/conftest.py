"""Shared pytest configuration: the ``gpu`` marker and common fixtures."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def gemma():
    """GEMMA reference outputs shipped with jamma's test-suite (committed as npz)."""
    return dict(np.load(GOLDEN / "gemma_fixtures.npz"))


@pytest.fixture(scope="session")
def ref_lik():
    """Outputs of jamma's own NumPy likelihood module on the gemma_synthetic cohort."""
    return dict(np.load(GOLDEN / "reference_likelihood.npz"))


@pytest.fixture(scope="session")
def gemma_geno(gemma):
    from oracle.plink import decode_packed

    return decode_packed(gemma["packed"], int(gemma["n"]))
