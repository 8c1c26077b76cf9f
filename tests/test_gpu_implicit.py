"""hotspin's implicit solvers on the device: solver/am12 (adaptive Adams-Moulton 1-2,
solve_am01.go:45-318) and solver/bdf-euler (fixed-step backward Euler,
solve_euler_backward.go:29-91), against the FP64 oracle's restatement, without a thermal
field.  The launch sequence itself is checked step by step on the CPU
(tests/test_control_rules.py); here the FP32 kernels run it.
"""
import numpy as np
import pytest

from hotspin_b200.sim import Batch, Simulation
from oracle import fields as F
from oracle.model import Model, Spec
from oracle.solvers import Integrator
from tests.gpu_util import rel_err

pytestmark = pytest.mark.gpu

MS = 8e5
LEX = float(np.sqrt(2 * 1.3e-11 / (F.MU0 * MS * MS)))
LLG = dict(size=(1, 16, 32), cellsize=(3e-9, 3.9e-9, 3.9e-9), msat0T0=MS, lex=LEX,
           gamma_ll=F.GAMMA0 / (1 + 0.02 ** 2), alpha=(0.02,) * 3, b_ext=(0.0, 0.012, 0.016), demag=True,
           normalize=True)
# the reference's laser example in miniature (examples/laser-demag.py runs solver/am12)
TTM = dict(size=(2, 16, 32), cellsize=(4e-9,) * 3, msat0T0=MS, lex=LEX, gamma_ll=F.GAMMA0 / (1 + 0.02 ** 2),
           alpha=(0.02,) * 3, b_ext=(0.02, 0.0, 0.0), demag=True, llb=True, tc=630.0, spin_j=0.5,
           n_spins=MS / (2 * F.MUB * 0.5), temperature=300.0, ttm=True, gamma_e=700.0, c_l=3e6, g_ep=6e17,
           k_e=90.0, k_l=0.0, laser_p0=5e20, laser_t0=5e-14, laser_fwhm=1e-13, laser_sigma=40e-9)


def _start(kw):
    size = kw["size"]
    if not kw.get("ttm"):
        return {"m": np.stack([np.zeros(size), np.full(size, 2 ** -0.5), np.full(size, 2 ** -0.5)])}
    rng = np.random.default_rng(3)
    th = np.deg2rad(5.0) * rng.random(size)
    ph = 2 * np.pi * rng.random(size)
    me = F.equilibrium_m(300.0, 630.0, 0.5)
    m = me * np.stack([np.cos(th), np.sin(th) * np.sin(ph), np.sin(th) * np.cos(ph)])
    return {"m": m, "Te": np.full(size, 300.0), "Tl": np.full(size, 300.0)}


@pytest.mark.parametrize("case", ["llg", "llg-1e-5", "ttm"])
def test_am12_matches_oracle(cuda, case):
    kw = TTM if case == "ttm" else LLG
    y0 = _start(kw)
    keys = list(y0)
    # the LLG film at the reference's default tolerances for m and at 1e-5 / 1e-5; the
    # two-temperature case at the laser example's 1e-5
    ab = {"m": 1e-4 if case == "llg" else 1e-5, "Te": 1e-2, "Tl": 1e-2}
    rl = {"m": 1e-3 if case == "llg" else 1e-5, "Te": 1e-5, "Tl": 1e-5}
    t_end = 0.3e-12
    it = Integrator(Model(Spec(**kw)), y0, "am12", 1e-17, mindt=1e-22, maxdt=1e-12,
                    maxabserr={k: ab[k] for k in keys}, maxrelerr={k: rl[k] for k in keys})
    it.run_until(t_end)
    with Simulation(**kw, solver="am12", dt=1e-17, mindt=1e-22, maxdt=1e-12, maxerr=(ab["m"], ab["Te"], ab["Tl"]),
                    maxrelerr=(rl["m"], rl["Te"], rl["Tl"])) as sim:
        for k, v in y0.items():
            sim.set(k, v)
        sim.run_until(t_end)
        st = sim.status()
        m = sim.get("m")
        T = sim.get("Te") if kw.get("ttm") else None
    want = F.normalize(it.y["m"]) if kw.get("normalize") else it.y["m"]
    dm = float(np.abs(m - want).max())
    print("\n[am12] %s steps %d (oracle %d) max|dm| %.2e" % (case, st["steps"], it.step_count, dm))
    assert st["t"] == pytest.approx(t_end, rel=1e-9)
    assert abs(st["steps"] - it.step_count) <= max(1, it.step_count // 50)
    assert dm < 1e-5
    if T is not None:
        assert rel_err(T, it.y["Te"]) < 1e-5


@pytest.mark.parametrize("case", ["llg", "ttm"])
def test_bdf_euler_matches_oracle(cuda, case):
    kw = LLG if case == "llg" else TTM
    y0 = _start(kw)
    tol = 1e-4 if case == "llg" else 1e-6
    it = Integrator(Model(Spec(**kw)), y0, "bdf_euler", 5e-16, max_iter=8, max_iter_err=tol)
    it.run_steps(40)
    with Simulation(**kw, solver="bdf-euler", dt=5e-16, maxerr=(tol, 0.0, 0.0), max_iter=8) as sim:
        for k, v in y0.items():
            sim.set(k, v)
        sim.step(40)
        st = sim.status()
        m = sim.get("m")
        T = sim.get("Te") if kw.get("ttm") else None
    assert st["steps"] == 40 and st["status"] == 0
    assert float(np.abs(m - it.y["m"]).max()) < 1e-5
    if T is not None:
        assert rel_err(T, it.y["Te"]) < 1e-5


def test_bdf_euler_unconverged_iteration_stops_the_run(cuda):
    from hotspin_b200 import _lib
    kw = LLG
    with Simulation(**kw, solver="bdf-euler", dt=5e-14, maxerr=(1e-12, 0.0, 0.0), max_iter=1) as sim:
        sim.set("m", _start(kw)["m"])
        rc = sim._lib.hsb_sim_step(sim._h, 2)
        assert rc == 6, sim._lib.hsb_last_error()       # HSB_ERR_SOLVER
        assert sim.status()["status"] & 4


def test_am12_batch_slot_matches_plain_handle(cuda):
    kw = dict(LLG, size=(1, 16, 32), solver="am12", dt=1e-17, mindt=1e-22, maxdt=1e-12, maxerr=(1e-5, 0, 0),
              maxrelerr=(1e-5, 0, 0), rtol=1e-5)
    cls = {k: kw[k] for k in ("size", "cellsize", "solver", "rtol", "demag", "dt", "msat0T0", "gamma_ll", "maxerr",
                              "maxrelerr")}
    y0 = _start(kw)["m"]
    with Batch(2, **cls) as b:
        b.admit(0, y0, 0.1e-12, **kw)
        for _ in range(100000):
            b.launch(1)
            while not b.poll():
                pass
            if not b.slot_status(0)["active"]:
                break
        mb, sb = b.slot_get(0, "m"), b.slot_status(0)
    with Simulation(**kw) as sim:
        sim.set("m", y0)
        sim.run_until(0.1e-12)
        m, st = sim.get("m"), sim.status()
    assert sb["steps"] == st["steps"]
    assert float(np.abs(mb - m).max()) <= 1e-6


def test_am12_matches_reference_kernels(cuda):
    """The reference's own kernels (oracle/_ref) stepped by the replay of solve_am01.go."""
    from oracle import replay
    if not replay.available():
        pytest.skip("oracle/_ref/libhotspin.so not built (needs the reference sources)")
    kw = dict(LLG, size=(1, 16, 32))
    y0 = _start(kw)
    ref = replay.RefSim(kw, dt=1e-17, mindt=1e-22, maxdt=1e-12)
    ref.set("m", y0["m"])
    t_end = 0.2e-12
    while t_end - ref.t > 1e-6 * ref.dt:
        ref.dt = min(ref.dt, t_end - ref.t)
        ref.step_am12({"m": 1e-4}, {"m": 1e-3})
    with Simulation(**kw, solver="am12", dt=1e-17, mindt=1e-22, maxdt=1e-12, maxerr=(1e-4, 0.0, 0.0),
                    maxrelerr=(1e-3, 0.0, 0.0)) as sim:
        sim.set("m", y0["m"])
        sim.run_until(t_end)
        st = sim.status()
        m = sim.get("m")
    assert st["t"] == pytest.approx(t_end, rel=1e-9)
    assert abs(st["steps"] - ref.steps) <= max(1, ref.steps // 50)
    assert float(np.abs(m - ref.get("m")).max()) < 1e-5
