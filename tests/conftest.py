import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the kernels)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the library and the oracle in-tree once per session (no-op when fresh)."""
    from voxelcraft_menu_b200 import build as b
    from oracle import build as ob
    if not os.environ.get("VM_SKIP_BUILD"):
        b.build()
        ob.build()


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
