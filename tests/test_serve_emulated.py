"""The continuous-batching loop (hotspin_b200/serve.py) end to end on the emulated kernels
(tests/emu): a short stream of mixed-size requests served in batches gives, request by
request, the plain single-simulation path's result bit for bit and the same step counts."""
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
import numpy as np
from hotspin_b200 import serve
reqs = serve.make_requests(n=5, rate=1000.0, seed=4, t_end=1e-13, sides=(32, 64), layers=(1,))
srv = serve.Server()
res = srv.run(reqs, realtime=False)
classes = len(srv.classes)
srv.close()
seq, service, setup = serve.run_sequential(reqs)
dm = max(float(np.abs(res[k].m - seq[k].m).max()) for k in res)
same = sum(int(res[k].steps == seq[k].steps) for k in res)
print("RESULT", len(res), classes, dm, same)
"""


def test_batched_serving_matches_the_plain_path_on_the_emulated_kernels():
    if not shutil.which("g++"):
        pytest.skip("g++ is not available")
    p = subprocess.run([sys.executable, "-c", SCRIPT % ROOT], cwd=ROOT, capture_output=True, text=True, timeout=1200)
    assert p.returncode == 0, p.stderr[-3000:]
    line = [l for l in p.stdout.splitlines() if l.startswith("RESULT")][-1].split()
    n, classes, dm, same = int(line[1]), int(line[2]), float(line[3]), int(line[4])
    assert n == 5 and classes >= 2
    assert dm == 0.0
    assert same == n
