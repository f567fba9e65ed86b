import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
if str(ROOT / "tests") not in sys.path:
    sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")


def _cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    """torch with a CUDA device; GPU tests skip (with a reason) on a CPU-only machine."""
    if not _cuda_available():
        pytest.skip("no CUDA device")
    import torch

    from su3_ma_gauge_gpu_b200 import lib

    lib()  # fails loudly if libgfix.so is missing
    return torch
