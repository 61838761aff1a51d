import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "procedural-generation_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def cuda():
    import torch

    # GPU tests fail rather than skip without a device: a skipped parity test
    # must never read as a pass on a machine with a GPU
    assert torch.cuda.is_available(), "this test needs a CUDA device"
    return torch.device("cuda:0")
