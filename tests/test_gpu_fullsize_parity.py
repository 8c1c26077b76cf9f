"""T = 0 parity at full size against the reference's own FP64 kernels.

The reference's CUDA library (oracle/_ref/libhotspin.so, built from its sources) driven by
the replay of the Go call sequence (oracle/replay.py, FP64, cuFFT) is the FP64 oracle at
sizes the NumPy oracle cannot reach.  Both runs start from the same state, use the same
DP45 rule at rtol 1e-5 and stop at the same time; thermal fields are off (T = 0 parity; the
bath temperature still sets the LLB and two-temperature physics).

* the two-temperature + LLB workload of the benchmark, 512 x 512 x 4 cells of 4 nm with the
  laser pulse, to 20 ps;
* the FePt-like LLB workload, 256 x 256 x 8 cells of 2 nm at 300 K, to 2 ps (its longitudinal
  relaxation needs femtosecond steps; 2 ps keeps the reference's replay near a minute).
"""
import math

import numpy as np
import pytest

from hotspin_b200.sim import Simulation
from oracle import fields as F
from oracle import replay
from tests.gpu_util import rel_err

pytestmark = [pytest.mark.gpu, pytest.mark.late]

MU0 = 4e-7 * math.pi


def _run_ref(kw, state, t_end, dt0):
    sim = replay.RefSim(kw, dt=dt0, rtol=1e-5, mindt=1e-20, maxdt=1e-13)
    for k, v in state.items():
        sim.set(k, v)
    while t_end - sim.t > 1e-6 * sim.dt:
        sim.dt = min(sim.dt, t_end - sim.t)
        sim.step()
    return sim


def _run_ours(kw, state, t_end, dt0):
    with Simulation(**kw, solver="dp45", dt=dt0, rtol=1e-5, mindt=1e-20, maxdt=1e-13) as sim:
        for k, v in state.items():
            sim.set(k, v)
        sim.run_until(t_end)
        out = {k: sim.get(k) for k in state}
        out["status"] = sim.status()
    return out


@pytest.fixture(scope="module")
def ref(cuda):
    if not replay.available():
        pytest.skip("oracle/_ref/libhotspin.so not built (needs the reference sources)")
    return replay


def test_ttm_llb_laser_512x512x4_to_20ps(ref):
    import bench
    kw = dict(bench.workload(), thermal=False)
    state = bench.initial_state(kw, F.equilibrium_m(300.0, kw["tc"], kw["spin_j"]))
    t_end = 20e-12
    want = _run_ref(kw, state, t_end, 2e-16)
    got = _run_ours(kw, state, t_end, 2e-16)
    dm = float(np.abs(got["m"] - want.get("m")).max())
    dT = rel_err(got["Te"], want.get("Te"))
    st = got["status"]
    print("\n[full size TTM+LLB 20 ps] steps %d (reference kernels %d)  max|dm| %.2e  rel max|dTe| %.2e"
          % (st["steps"], want.steps, dm, dT))
    assert st["t"] == pytest.approx(t_end, rel=1e-9)
    # FP32 and FP64 error norms take slightly different steps near the tolerance (a reduced grid
    # of the same workload on the emulated kernels: 294 against 290 steps over 5 ps)
    assert abs(st["steps"] - want.steps) <= max(4, want.steps // 20)
    assert dm <= 1e-5
    assert dT <= 1e-5


def test_llb_fept_256x256x8_to_2ps(ref):
    size = (8, 256, 256)
    ms = 1.1e6
    kw = dict(size=size, cellsize=(2e-9,) * 3, msat0T0=ms, lex=math.sqrt(2 * 1e-11 / (MU0 * ms * ms)),
              gamma_ll=2.211e5, alpha=(0.1,) * 3, ku=7e6, anis_u=(1.0, 0.0, 0.0), demag=True, llb=True, tc=700.0,
              spin_j=0.5, n_spins=ms / (2 * F.MUB * 0.5), temperature=300.0, thermal=False)
    rng = np.random.default_rng(2)
    th = np.deg2rad(5.0) * rng.random(size)
    ph = 2 * np.pi * rng.random(size)
    me = F.equilibrium_m(300.0, 700.0, 0.5)
    state = {"m": me * np.stack([np.cos(th), np.sin(th) * np.sin(ph), np.sin(th) * np.cos(ph)])}
    t_end = 2e-12
    want = _run_ref(kw, state, t_end, 1e-16)
    got = _run_ours(kw, state, t_end, 1e-16)
    dm = float(np.abs(got["m"] - want.get("m")).max())
    st = got["status"]
    print("\n[full size LLB 256x256x8 2 ps] steps %d (reference kernels %d)  max|dm| %.2e"
          % (st["steps"], want.steps, dm))
    assert st["t"] == pytest.approx(t_end, rel=1e-9)
    assert dm <= 1e-5
