import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls the engine through the C ABI")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not _has_gpu():
        pytest.skip("no CUDA device")
    return 0


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the engine library and the oracle if they are missing (the
    build script runs standalone: importing the package needs the library)."""
    import subprocess
    subprocess.run([sys.executable, os.path.join(ROOT, "mercurydpm_fork_b200", "build.py")], check=True,
                   stdout=subprocess.DEVNULL)
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
