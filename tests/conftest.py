import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the native CUDA path")
    config.addinivalue_line("markers", "slow: longer CPU test")


def _build():
    if not os.path.exists(os.path.join(ROOT, "qcmaquis_b200", "libqcm_b200.so")):
        subprocess.run(["make", "-C", os.path.join(ROOT, "qcmaquis_b200", "csrc"), "-j8"], check=True,
                       stdout=subprocess.DEVNULL)
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, stdout=subprocess.DEVNULL)


_build()


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_ctx():
    if not has_gpu():
        pytest.fail("GPU test requested but no CUDA device is visible")
    from qcmaquis_b200.heff import Context
    return Context(0)
