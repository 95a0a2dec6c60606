"""Shared test set-up: the ``gpu`` marker and import paths.

``-m "not gpu"`` runs the oracle-against-golden pins, the host planner and the C-ABI
symbol checks on a CPU-only machine; ``-m gpu`` runs the parity tests through the CUDA
library on a B200.
"""

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "tenet-py_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def has_cuda() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def golden_dir() -> Path:
    return GOLDEN
