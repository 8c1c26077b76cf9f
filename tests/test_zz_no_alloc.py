"""hsb_average_m_noalloc: the allocation-free variant of the handle's average-of-m reduction.

Callers that own every device buffer (hotspin's Go layer allocates all device memory
itself; other hosts manage GPU memory through their own pools) cannot have the library
call cudaMalloc.  This entry point keeps its reduction scratch in a static device array;
here its output is checked against hsb_sim_average_m, which runs the same reduction on the
simulation handle's own allocated scratch, on two calls in a row (the shared scratch and
its counter must be reusable).  Kept in a file of its own, collected last.
"""
import ctypes

import numpy as np
import pytest

from hotspin_b200 import _lib
from hotspin_b200.sim import Simulation

pytestmark = pytest.mark.gpu


def test_noalloc_average_matches_handle(cuda):
    torch = cuda
    lib = _lib.load()
    size = (2, 48, 80)
    rng = np.random.default_rng(2024)
    with Simulation(size=size, cellsize=(1e-9,) * 3, msat0T0=8e5, solver="rk4", dt=1e-15) as sim:
        for call in range(2):
            m = rng.normal(size=(3,) + size)
            m[2] += 0.3 * (call + 1)
            sim.set("m", m)
            want = sim.average_m()                       # existing entry point (handle scratch)
            m32 = torch.from_numpy(m.astype(np.float32)).cuda().contiguous()
            out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
            rc = lib.hsb_average_m_noalloc(ctypes.c_void_p(m32.data_ptr()), m32[0].numel(),
                                           ctypes.c_void_p(out.data_ptr()), None)
            _lib.check(rc, "hsb_average_m_noalloc")
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert np.allclose(got, want, rtol=1e-12, atol=1e-15), (call, got, want)


def test_noalloc_rejects_oversize(cuda):
    torch = cuda
    lib = _lib.load()
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    m = torch.zeros(3, dtype=torch.float32, device="cuda")
    rc = lib.hsb_average_m_noalloc(ctypes.c_void_p(m.data_ptr()), (1 << 28) + 1, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1 and b"2^28" in lib.hsb_last_error()
    rc = lib.hsb_average_m_noalloc(ctypes.c_void_p(m.data_ptr()), 0, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1
