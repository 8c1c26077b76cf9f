"""Small standalone workloads for profiling the kernels (e.g. under ncu).

    python -m hotspin_b200.profile demag [N0 N1 N2]   # one demag plan, 3 + 11 convolutions
    python -m hotspin_b200.profile sim                # the bench simulation: 2 steps + 2 profiled attempts

Both print the per-kernel device times measured with CUDA events.
"""
import ctypes
import os
import sys

import numpy as np


def demag(size):
    import torch
    from . import _lib
    from .sim import demag_plan
    plan = demag_plan(size, (4e-9,) * 3, (0, 0, 0))
    lib = _lib.load()
    m = torch.randn((3,) + tuple(size), device="cuda", dtype=torch.float32)
    H = torch.empty_like(m)
    for _ in range(3):
        _lib.check(lib.hsb_demag_field(plan, ctypes.c_void_p(m.data_ptr()), None, 8e5,
                                       ctypes.c_void_p(H.data_ptr()), None), "hsb_demag_field")
    ms = (ctypes.c_double * 3)()
    _lib.check(lib.hsb_demag_profile(plan, ctypes.c_void_p(m.data_ptr()), None, 8e5, ctypes.c_void_p(H.data_ptr()),
                                     None, 10, ms), "hsb_demag_profile")
    torch.cuda.synchronize()
    print("demag", tuple(size), "ms x-fwd / y-z / x-inv", [round(x, 5) for x in ms])
    lib.hsb_demag_plan_destroy(plan)


def sim():
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from .sim import Simulation
    kw = bench.workload()
    st0 = bench.initial_state(kw)
    s = Simulation(**kw, solver="dp45", dt=2e-16, rtol=1e-5, mindt=1e-20, maxdt=1e-13)
    for k, v in st0.items():
        s.set(k, v)
    s.step(2)
    out = (ctypes.c_double * 7)()
    s._lib.hsb_sim_profile(s._h, 2, out)
    print("attempt ms: stage %.4f x-fwd %.4f y-z %.4f x-inv %.4f other %.4f launches %d" % tuple(out[:6]))
    s.close()


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "demag"
    if what == "demag":
        size = tuple(int(x) for x in sys.argv[2:5]) if len(sys.argv) >= 5 else (4, 512, 512)
        demag(size)
    else:
        sim()
