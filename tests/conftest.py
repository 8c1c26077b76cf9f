import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_addoption(parser):
    parser.addoption("--emulate-cuda", action="store_true",
                     help="run the gpu tests on the library's kernels built for the CPU emulation of CUDA "
                          "(tests/emu); tests of the reference's CUDA library are skipped")
    parser.addoption("--emulate-reference", action="store_true",
                     help="with --emulate-cuda: build the reference's own kernel library for the emulation "
                          "(oracle/ref_emu.py) and let the replay of hotspin's call sequence drive it; runs "
                          "every kernel in reverse scheduling order, which the reference's warp-synchronous "
                          "max reductions need there")
    parser.addoption("--replay-dropins", action="store_true",
                     help="with --emulate-cuda: let the replay of hotspin's call sequence (oracle/replay.py) "
                          "drive the product's FP64 drop-ins in place of the reference's library, to check "
                          "the replay's solver logic and the tests built on it (not the reference's kernels)")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU test")
    config.addinivalue_line("markers", "late: long-horizon or statistical gpu test, run after the others")
    if config.getoption("--emulate-cuda"):
        if config.getoption("--emulate-reference"):
            os.environ["HSBEMU_ORDER"] = "reverse"      # read by both emulated runtimes at first use
        use_emulated_library(config.getoption("--replay-dropins"))
        if config.getoption("--emulate-reference"):
            import oracle.replay
            from oracle import ref_emu
            if ref_emu.available():
                oracle.replay.REF_LIB = ref_emu.build()
                oracle.replay.available = lambda: True


def use_emulated_library(replay_dropins=False):
    """Bind tests/emu's build of the library (same C ABI and signatures) as the handle the
    package's bindings use in this test process, in place of libhsb200.so."""
    import ctypes
    from tests.emu import build as emu_build
    from hotspin_b200 import _lib
    # HSBEMU_ASAN=1 (with the process started under LD_PRELOAD of libasan): the AddressSanitizer
    # build, which reports any out-of-bounds access of a kernel to host memory
    lib = ctypes.CDLL(emu_build.build(asan=os.environ.get("HSBEMU_ASAN") == "1"))
    for name, (res, args) in _lib._SIGS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib._lib = lib
    import oracle.replay
    if replay_dropins:                           # the drop-ins stand in for the reference's library
        oracle.replay.REF_LIB = lib._name
        oracle.replay.available = lambda: True
    else:
        oracle.replay.available = lambda: False  # the reference's library needs a real GPU
    _torch_device_memory_on_the_host()


def _torch_device_memory_on_the_host():
    """Under the emulation every device pointer is a host pointer: torch's "cuda" tensors of
    the tests become CPU tensors (Tensor.cuda() returns a copy, as the transfer does,
    device="cuda" means the CPU, synchronisation is a no-op)."""
    import torch
    torch.Tensor.cuda = lambda self, *a, **k: self.clone()
    to = torch.Tensor.to

    def to_host(self, *a, **k):
        a = tuple("cpu" if str(x).startswith("cuda") else x for x in a)
        if str(k.get("device", "")).startswith("cuda"):
            k["device"] = "cpu"
        return to(self, *a, **k)
    torch.Tensor.to = to_host
    torch.cuda.synchronize = lambda *a, **k: None

    class _Stream:
        cuda_stream = 0

        def synchronize(self):
            pass
    torch.cuda.current_stream = lambda *a, **k: _Stream()
    torch.cuda.ExternalStream = lambda *a, **k: _Stream()
    torch.cuda.set_device = lambda *a, **k: None

    class _Event:            # host clock: every emulated launch has finished when it returns
        def __init__(self, enable_timing=False, **k):
            self.t = None

        def record(self, stream=None):
            import time
            self.t = time.perf_counter()

        def synchronize(self):
            pass

        def elapsed_time(self, other):
            return (other.t - self.t) * 1e3
    torch.cuda.Event = _Event
    empty = torch.empty

    def empty_unpinned(*a, **k):
        k.pop("pin_memory", None)            # page-locking needs the CUDA driver
        if str(k.get("device", "")).startswith("cuda"):
            k["device"] = "cpu"
        return empty(*a, **k)
    torch.empty = empty_unpinned
    for name in ("full", "zeros", "ones", "tensor", "randn", "rand", "arange", "zeros_like",
                 "empty_like", "full_like", "ones_like"):
        f = getattr(torch, name)

        def on_host(*a, _f=f, **k):
            if str(k.get("device", "")).startswith("cuda"):
                k["device"] = "cpu"
            return _f(*a, **k)
        setattr(torch, name, on_host)


@pytest.fixture(scope="session")
def cuda(request):
    """torch with a CUDA device; the gpu-marked tests use it for device buffers only.  Under
    --emulate-cuda, torch with its "cuda" tensors in host memory."""
    import torch
    if request.config.getoption("--emulate-cuda"):
        return torch
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


def pytest_collection_modifyitems(config, items):
    """Long-horizon and statistical gpu tests (marked `late`) run after the others, so that a
    run stopping at its first failure has checked everything else; tests/test_zz_no_alloc.py
    stays last."""
    def rank(it):
        if os.path.basename(str(it.fspath)) == "test_zz_no_alloc.py":
            return 2
        return 1 if it.get_closest_marker("late") else 0
    items[:] = sorted(items, key=rank)     # stable: the file order holds within each group
