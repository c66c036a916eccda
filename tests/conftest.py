import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _ensure_native():
    """Build the in-tree library and the oracle if they are missing (both are
    cheap; nvcc and gcc exist wherever the tests run)."""
    from cpp_projects_b200 import build as b
    if not b.LIB.exists():
        b.build()
    from oracle import pyoracle
    if not (pyoracle.HERE / "liboracle.so").exists():
        pyoracle.build()


_ensure_native()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
