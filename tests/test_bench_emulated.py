"""bench.py's own logic (warm-up, checkpointed repetitions of exactly K steps, per-kernel
profile and roofline, end-to-end run through the C ABI, the JSON line) on the emulated kernels
(tests/emu) at a reduced grid: the line has every key of the contract and the repetitions
repeat the same trajectory.  Timings here are the emulator's and mean nothing."""
import json
import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys
sys.path.insert(0, %r)
import tests.conftest as C
C.use_emulated_library()
import bench
full = bench.workload
def small():
    kw = full()
    kw["size"] = (2, 32, 32)
    kw["laser_sigma"] = 40e-9
    return kw
bench.workload = small
sys.argv = ["bench.py", "--steps", "4", "--warmup", "3", "--no-serving", "--no-configs", "--no-cpu-baseline",
            "--min-reps", "2", "--min-timed-s", "0"]
bench.main()
"""


def test_bench_line_on_the_emulated_kernels():
    if not shutil.which("g++"):
        pytest.skip("g++ is not available")
    p = subprocess.run([sys.executable, "-c", SCRIPT % ROOT], cwd=ROOT, capture_output=True, text=True, timeout=1200)
    assert p.returncode == 0, p.stderr[-3000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "roofline", "gpu_launches", "e2e", "clocks", "timing"):
        assert k in line, k
    assert line["steps"] == 4 and line["warmup"] == 3 and line["n_gpus"] == 1
    assert line["timing"]["identical_repetitions"] is True
    assert line["gpu_launches"] > 0 and line["value"] > 0
    for k in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert k in line["roofline"], k
    for k in ("value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"):
        assert k in line["e2e"], k
    assert line["e2e"]["h2d_bytes_per_step"] > 0 and line["e2e"]["d2h_bytes_per_step"] > 0
    assert line["progress"]["attempts"] >= 4


REF_SCRIPT = r"""
import os, sys
os.environ["HSBEMU_ORDER"] = "reverse"
sys.path.insert(0, %r)
import tests.conftest as C
C.use_emulated_library()
import oracle.replay
from oracle import ref_emu
oracle.replay.REF_LIB = ref_emu.build()
oracle.replay.available = lambda: True
import bench
full = bench.workload
def small():
    kw = full()
    kw["size"] = (2, 32, 32)
    kw["laser_sigma"] = 40e-9
    return kw
bench.workload = small
sys.argv = ["bench.py", "--impl", "reference", "--steps", "3", "--warmup", "3"]
bench.main()
"""


def test_reference_arm_line_on_the_emulated_reference_kernels():
    """bench.py --impl reference (the replay of hotspin's call sequence on the reference's own
    kernels, oracle/ref_emu.py's build for the emulation): the line carries the contract's keys
    and the same config as the product's line."""
    if not shutil.which("g++"):
        pytest.skip("g++ is not available")
    from oracle import ref_emu
    if not ref_emu.available():
        pytest.skip("no reference checkout")
    p = subprocess.run([sys.executable, "-c", REF_SCRIPT % ROOT], cwd=ROOT, capture_output=True, text=True,
                       timeout=1200)
    assert p.returncode == 0, p.stderr[-3000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "unavailable" not in line
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["steps"] == 3 and line["warmup"] == 3 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
