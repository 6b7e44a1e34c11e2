import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA kernels through the C ABI")
    # the library is built in-tree; build it on first use where nvcc exists and it is missing
    lib = ROOT / "ghex_b200" / "libghex_b200.so"
    if not lib.exists():
        from ghex_b200 import build as _build
        _build.build()


@pytest.fixture(scope="session")
def cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch.device("cuda", 0)
