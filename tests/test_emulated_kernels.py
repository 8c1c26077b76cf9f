"""The library's kernels, unchanged, on the CPU emulation of CUDA (tests/emu), against the oracle.

A selection of the gpu tests -- the ones whose code paths have the most host logic around the
kernels: the reference's solvers (rk12, am12, bdf-euler), the optional LLBar terms, the Newell
tensor, grids embedded in a power-of-two demag grid, failure handling (non-finite states,
unreachable tolerances, checkpoints, batch slot release), the FP64 FFT plan and the FP64 drop-ins
under the Go call sequence -- runs in a child pytest with --emulate-cuda, where the library is the product's
CUDA source built as host C++ against the emulated runtime (every CUDA thread a fiber, block and
warp barriers, graph capture and replay).  The full gpu suite runs the same way with
``python -m pytest tests -m gpu --emulate-cuda`` (tens of minutes).
"""
import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SELECTION = [
    "tests/test_gpu_failures.py",
    "tests/test_gpu_newell.py",
    "tests/test_gpu_rk12.py::test_rk12_matches_oracle",
    "tests/test_gpu_implicit.py::test_am12_matches_oracle[llg]",
    "tests/test_gpu_implicit.py::test_am12_matches_oracle[llg-1e-5]",
    "tests/test_gpu_implicit.py::test_bdf_euler_matches_oracle[llg]",
    "tests/test_gpu_implicit.py::test_bdf_euler_unconverged_iteration_stops_the_run",
    "tests/test_gpu_implicit.py::test_am12_batch_slot_matches_plain_handle",
    "tests/test_gpu_sim.py::test_rhs_matches_oracle",
    "tests/test_gpu_sim.py::test_second_order_relaxation_terms",
    "tests/test_gpu_sim.py::test_nonlocal_relaxation_term",
    "tests/test_gpu_demag.py::test_demag_on_grids_that_do_not_pad_to_powers_of_two",
    "tests/test_gpu_xfftplan.py",
]


REPLAY_SELECTION = [
    "tests/test_gpu_reference_replay.py",
    "tests/test_gpu_rk12.py::test_rk12_matches_reference_kernels",
    "tests/test_gpu_implicit.py::test_am12_matches_reference_kernels",
    "tests/test_gpu_dropin_replay.py",
]


def _run(args):
    """A child pytest on the emulated library (built here first, so its workers reuse it)."""
    from tests.emu import build as emu_build
    emu_build.build()
    import importlib.util
    workers = ["-n", str(min(4, os.cpu_count() or 1))] if importlib.util.find_spec("xdist") else []
    cmd = [sys.executable, "-m", "pytest", "-m", "gpu", "--emulate-cuda", "-q", "-p", "no:cacheprovider"] + workers + args
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=1800)
    return p, "\n".join(p.stdout.splitlines()[-30:])


def test_replay_tests_on_the_reference_kernels():
    """oracle/replay.py's restatement of hotspin's solver loops (dp45, rk12, am12) on the
    reference's own kernels built for the emulation (oracle/ref_emu.py), and the tests that
    compare the product with them: the product's FP32 handle, its FP64 drop-ins under the Go call
    sequence and the FP64 oracle against the reference's kernels.  Without the reference
    checkout, the product's drop-ins stand in for the reference's library (a check of the
    replay's logic only)."""
    if not shutil.which("g++"):
        pytest.skip("g++ is not available")
    from oracle import ref_emu
    if ref_emu.available():
        ref_emu.build()              # here, so the child's workers reuse it
        p, tail = _run(["--emulate-reference"] + REPLAY_SELECTION)
    else:
        p, tail = _run(["--replay-dropins"] + REPLAY_SELECTION[:3])
    assert p.returncode == 0, tail
    assert " passed" in tail and "failed" not in tail and "skipped" not in tail, tail


def test_selected_gpu_tests_pass_on_the_emulated_kernels():
    if not shutil.which("g++"):
        pytest.skip("g++ is not available")
    p, tail = _run(SELECTION)
    assert p.returncode == 0, tail
    assert " passed" in tail and "failed" not in tail, tail
