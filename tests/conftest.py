"""Shared test configuration.

Tests marked `gpu` need a B200 and call the product through its C ABI;
everything else runs on the CPU (oracle against golden vectors and known
answers, host logic, library loading and exports)."""

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ctx():
    import heddle_b200 as hb

    c = hb.Context(0)
    yield c
    c.close()
