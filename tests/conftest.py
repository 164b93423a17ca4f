import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs through the C ABI")


@pytest.fixture(scope="session", autouse=True)
def _native_build():
    """Make sure the in-tree libraries exist (rebuilds only what is stale)."""
    from hacapk_hmvm_b200 import build

    build.build_all()
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True,
                   stdout=subprocess.DEVNULL)
    yield


def cuda_ok() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not cuda_ok():
        pytest.fail("a CUDA device is required for tests marked gpu")
    import torch

    return torch.device("cuda:0")


_REPORT = []


@pytest.fixture(scope="session")
def report():
    """Lines shown in the terminal summary: the measured relative errors of
    the parity tests at configuration size, beside their bounds."""
    return _REPORT


def pytest_terminal_summary(terminalreporter):
    if _REPORT:
        terminalreporter.write_sep("-", "parity at configuration size (relative 2-norm error)")
        for line in _REPORT:
            terminalreporter.write_line(line)
