"""Test configuration: the ``gpu`` marker and shared fixtures.

``-m "not gpu"`` runs on any host (oracle, host logic, C-ABI symbols);
``-m gpu`` needs a CUDA device and runs the parity tests through the C ABI.
"""

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libgpe_ssf.so")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    from gpe_simulator_b200 import build
    build.build()
    torch.cuda.set_device(0)
    return torch.device("cuda:0")
