"""Large-instance precision study (the 1024x1024x32 LLG workload).

Plain LLG at T = 0, alpha 0.5, RK4 at 20 fs for 2000 steps.  The FP32 path runs the large
grid (1024x1024x32 cells of 2 nm, demag padded to 2048x2048x64, multi-pass FFT); the FP64
comparison runs the same sample at 256x256x8 cells of 8 nm on the reference's own kernels
(oracle/replay.py; the NumPy oracle needs hours at that size).  Both start from one seeded
random pattern defined on the coarse grid (seed 5), the fine grid from it upsampled (4x4x4 fine
cells per coarse cell).  Printed: max|dm| and mean|dm| of the fine result block-averaged onto
the coarse grid against the FP64 result and the relative difference of the total energies (a
discretisation difference as much as a precision one: 8 nm cells exceed the 5.7 nm exchange
length), and, to separate precision, the FP32 path on the coarse grid against the same FP64 run.
The relaxation from a random pattern passes through vortex annihilations whose outcome can
depend on rounding, so the numbers are reported, with only a sanity bound (1e-2) on the
same-grid energy.  Run with -s to see them.
"""
import math
import time

import numpy as np
import pytest

from hotspin_b200.sim import Simulation
from oracle import replay
from oracle.model import Model, Spec

pytestmark = [pytest.mark.gpu, pytest.mark.late]

MU0 = 4e-7 * math.pi


def test_config5_precision_study(cuda):
    if not replay.available():
        pytest.skip("oracle/_ref/libhotspin.so not built (the FP64 side runs the reference's kernels)")
    ms = 8e5
    base = dict(msat0T0=ms, lex=math.sqrt(2 * 1.3e-11 / (MU0 * ms * ms)), gamma_ll=2.211e5 / (1 + 0.25),
                alpha=(0.5,) * 3, demag=True, normalize=True)
    coarse, fine = (8, 256, 256), (32, 1024, 1024)
    rng = np.random.default_rng(5)
    mc = rng.normal(size=(3,) + coarse)
    mc /= np.sqrt((mc * mc).sum(0))
    mf = np.repeat(np.repeat(np.repeat(mc, 4, axis=1), 4, axis=2), 4, axis=3)
    nsteps, dt = 2000, 20e-15
    t0 = time.perf_counter()
    with Simulation(size=fine, cellsize=(2e-9,) * 3, solver="rk4", dt=dt, **base) as sim:
        sim.set("m", mf)
        sim.step(nsteps)
        m_fine = sim.get("m")
        e_fine = sim.energy()
    t_fine = time.perf_counter() - t0
    with Simulation(size=coarse, cellsize=(8e-9,) * 3, solver="rk4", dt=dt, **base) as sim:
        sim.set("m", mc)
        sim.step(nsteps)
        m_c32 = sim.get("m")
        e_c32 = sim.energy()
    kw = dict(size=coarse, cellsize=(8e-9,) * 3, **base)
    ref = replay.RefSim(kw, dt=dt)
    ref.set("m", mc)
    for _ in range(nsteps):
        ref.step_rk4()
    m64 = ref.get("m")
    e64 = Model(Spec(**kw)).energy({"m": m64})
    down = m_fine.reshape(3, coarse[0], 4, coarse[1], 4, coarse[2], 4).mean(axis=(2, 4, 6))
    down /= np.sqrt((down * down).sum(0))
    report = {
        "fine_fp32_seconds": round(t_fine, 1),
        "fine_vs_fp64_max_abs_dm": float(np.abs(down - m64).max()),
        "fine_vs_fp64_mean_abs_dm": float(np.abs(down - m64).mean()),
        "fine_vs_fp64_rel_energy": float(abs(e_fine - e64) / abs(e64)),
        "coarse_fp32_vs_fp64_max_abs_dm": float(np.abs(m_c32 - m64).max()),
        "coarse_fp32_vs_fp64_rel_energy": float(abs(e_c32 - e64) / abs(e64)),
    }
    print("\n[config-5 study]", report)
    assert np.isfinite(m_fine).all() and np.isfinite(e_fine)
    assert report["coarse_fp32_vs_fp64_rel_energy"] < 1e-2
