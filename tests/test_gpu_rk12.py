"""hotspin's adaptive Heun solver (solver/rk12, solve_rk12.go:91-214) on the device.

The device runs the attempt as two fused stages (Euler predictor with k0 = f(y0); Heun
corrector with the per-equation error dt max|k1 - k0|) and the step-size rule on the device
(hsb_rk12_rule).  Checked against the FP64 oracle's restatement, against the reference's own
kernels driven through the replay of the Go call sequence, through the script-API mirror and
in a batch, all without a thermal field (T = 0 parity at 1e-5).
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
# the standard-problem geometry of the reference's rk12 script (tests/stdproblem4-llbr-modular.py)
SP4 = dict(size=(1, 32, 128), cellsize=(3e-9, 125e-9 / 32, 500e-9 / 128), msat0T0=MS, lex=LEX,
           gamma_ll=F.GAMMA0 / (1 + 0.02 ** 2), alpha=(0.02,) * 3, b_ext=(0.0, 4.3e-3, -24.6e-3), demag=True,
           normalize=True)
TTM = dict(size=(2, 16, 32), cellsize=(4e-9,) * 3, msat0T0=MS, lex=LEX, gamma_ll=F.GAMMA0 / (1 + 0.02 ** 2),
           alpha=(0.02,) * 3, b_ext=(0.02, 0.0, 0.0), demag=True, llb=True, tc=630.0, spin_j=0.5,
           n_spins=MS / (2 * F.MUB * 0.5), temperature=300.0, ttm=True, gamma_e=700.0, c_l=3e6, g_ep=6e17,
           k_e=90.0, k_l=0.0, laser_p0=5e20, laser_t0=5e-14, laser_fwhm=1e-13, laser_sigma=40e-9)


def _sp4_start(size):
    return {"m": np.stack([np.zeros(size), np.full(size, 2 ** -0.5), np.full(size, 2 ** -0.5)])}


def _ttm_start(size):
    rng = np.random.default_rng(3)
    th = np.deg2rad(5.0) * rng.random(size)
    ph = 2 * np.pi * rng.random(size)
    me = F.equilibrium_m(300.0, 630.0, 0.5)
    m = me * np.stack([np.cos(th), np.sin(th) * np.sin(ph), np.sin(th) * np.cos(ph)])
    return {"m": m, "Te": np.full(size, 300.0), "Tl": np.full(size, 300.0)}


@pytest.mark.parametrize("case", ["sp4", "ttm"])
def test_rk12_matches_oracle(cuda, case):
    if case == "sp4":
        kw, y0, maxerr, t_end = SP4, _sp4_start(SP4["size"]), {"m": 1e-4}, 20e-12
    else:
        kw, y0, maxerr, t_end = TTM, _ttm_start(TTM["size"]), {"m": 1e-5, "Te": 0.5, "Tl": 0.5}, 0.5e-12
    it = Integrator(Model(Spec(**kw)), y0, "rk12", 1e-15, mindt=1e-20, maxdt=1e-12, maxerr=maxerr)
    it.run_until(t_end)
    me = (maxerr["m"], maxerr.get("Te", 0.0), maxerr.get("Tl", 0.0))
    with Simulation(**kw, solver="rk12", dt=1e-15, mindt=1e-20, maxdt=1e-12, maxerr=me) as sim:
        for k, v in y0.items():
            sim.set(k, v)
        sim.run_until(t_end)
        st = sim.status()
        m = sim.get("m")
        T = sim.get("Te") if kw.get("ttm") else None
    dm = float(np.abs(m - it.y["m"]).max())
    print("\n[rk12] %s steps %d (oracle %d) rejects %d (oracle %d) max|dm| %.2e"
          % (case, st["steps"], it.step_count, st["rejects"], it.bad_steps, dm))
    assert st["t"] == pytest.approx(t_end, rel=1e-9)
    assert abs(st["steps"] - it.step_count) <= max(1, it.step_count // 50)
    assert dm < 1e-5
    if T is not None:
        assert rel_err(T, it.y["Te"]) < 1e-5


def test_rk12_matches_reference_kernels(cuda):
    """The reference's own kernels (oracle/_ref) stepped by the replay of solve_rk12.go."""
    from oracle import replay
    if not replay.available():
        pytest.skip("oracle/_ref/libhotspin.so not built (needs the reference sources)")
    kw = dict(SP4, size=(1, 16, 64))
    y0 = _sp4_start(kw["size"])
    ref = replay.RefSim(kw, dt=1e-15, mindt=1e-20, maxdt=1e-12)
    ref.set("m", y0["m"])
    for _ in range(40):
        ref.step_rk12({"m": 1e-4})
    with Simulation(**kw, solver="rk12", dt=1e-15, mindt=1e-20, maxdt=1e-12, maxerr=(1e-4, 0.0, 0.0)) as sim:
        sim.set("m", y0["m"])
        sim.step(40)
        st = sim.status()
        m = sim.get("m")
    assert st["t"] == pytest.approx(ref.t, rel=1e-6)
    assert st["rejects"] == ref.rejects
    assert float(np.abs(m - ref.get("m")).max()) < 1e-5


def test_rk12_through_the_script_api(cuda):
    from hotspin_b200 import api
    e = api.new_engine()
    e.setgridsize(64, 16, 1)
    e.setcellsize(500e-9 / 128, 125e-9 / 32, 3e-9)
    for mod in ("exchange6", "demag", "zeeman", "llbar", "llbar/torque", "llbar/damping/nonconservative/00/local",
                "normalizer", "solver/rk12"):
        e.load(mod)
    e.setv("Msat0T0", MS)
    e.setv("lex", LEX)
    e.setv("α", [0.02] * 3)
    e.setv("γ_LL", F.GAMMA0 / (1 + 0.02 ** 2))
    e.setv("B_ext", [-24.6e-3, 4.3e-3, 0.0])
    e.setv("m_maxerror", 1e-4)
    e.setv("mindt", 1e-20)
    e.setv("maxdt", 1e-12)
    e.setv("dt", 1e-15)
    m_user = np.zeros((3, 64, 16, 1))
    m_user[0] = m_user[1] = 2 ** -0.5
    e.setarray("m", m_user)
    e.run(5e-12)
    assert e.getv("t") == pytest.approx(5e-12, rel=1e-9)
    got = e.getarray("m")
    kw = dict(SP4, size=(1, 16, 64))
    with Simulation(**kw, solver="rk12", dt=1e-15, mindt=1e-20, maxdt=1e-12, maxerr=(1e-4, 0.0, 0.0)) as sim:
        sim.set("m", _sp4_start(kw["size"])["m"])
        sim.run_until(5e-12)
        want = sim.get("m")
    # user order [x][y][z] components (x, y, z) vs program order
    from hotspin_b200.api import _to_user_vector
    np.testing.assert_array_equal(got, _to_user_vector(want))


def test_rk12_batch_slot_matches_plain_handle(cuda):
    kw = dict(SP4, size=(1, 16, 64), rtol=1e-4, maxerr=(1e-4, 0.0, 0.0), solver="rk12", dt=1e-15, mindt=1e-20,
              maxdt=1e-12)
    cls = {k: kw[k] for k in ("size", "cellsize", "solver", "rtol", "demag", "dt", "msat0T0", "gamma_ll", "maxerr")}
    y0 = _sp4_start(kw["size"])["m"]
    with Batch(2, **cls) as b:
        b.admit(1, y0, 3e-12, **kw)
        for _ in range(100000):
            b.launch(1)
            while not b.poll():
                pass
            if not b.slot_status(1)["active"]:
                break
        mb, sb = b.slot_get(1, "m"), b.slot_status(1)
    with Simulation(**kw) as sim:
        sim.set("m", y0)
        sim.run_until(3e-12)
        m, st = sim.get("m"), sim.status()
    assert sb["steps"] == st["steps"]
    assert float(np.abs(mb - m).max()) <= 1e-6
