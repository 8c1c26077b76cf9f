import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU test")


@pytest.fixture(scope="session")
def cuda():
    """torch with a CUDA device; the gpu-marked tests use it for device buffers only."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test selected but no CUDA device is visible")
    torch.cuda.init()
    return torch


@pytest.fixture(scope="session")
def hsb_lib():
    from hotspin_b200 import _lib
    return _lib.load()


@pytest.fixture(scope="session")
def host_rules(tmp_path_factory):
    """tests/native/rule_check.cu built with nvcc as host code: the device's shared step-control
    rules and Newell-tensor arithmetic, callable through ctypes without a GPU."""
    import ctypes
    import shutil
    import subprocess
    nvcc = "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else shutil.which("nvcc")
    if not nvcc:
        pytest.skip("nvcc is not available")
    out = str(tmp_path_factory.mktemp("rules") / "rule_check.so")
    cmd = [nvcc, "-x", "cu", "-std=c++17", "-O2", "-Xcompiler", "-fPIC", "-shared",
           "-I" + os.path.join(ROOT, "hotspin_b200", "csrc"), os.path.join(ROOT, "tests", "native", "rule_check.cu"),
           "-o", out]
    subprocess.run(cmd, check=True, capture_output=True)
    return ctypes.CDLL(out)
