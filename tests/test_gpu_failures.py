"""Failure handling of the handle and batch APIs, with every failure made on the host.

* a non-finite value planted in the host state (m or Te) before stepping ends the run with
  HSB_ERR_NONFINITE and status bit 1, for the fixed-step and the adaptive integrators, and a
  later step call refuses at once;
* an adaptive run whose tolerance cannot be met at the minimum step (rtol 1e-12, dt pinned to
  mindt) keeps stepping, as hotspin's rk12 does at its floor, and reports status bit 2;
* releasing a batch slot right behind a launched class graph leaves the other slots' results
  bit-identical to an undisturbed run;
* a checkpoint restored on the device repeats the original continuation bit for bit.
No kernel is made to fault: the bad value is ordinary input data.
"""
import ctypes

import numpy as np
import pytest

from hotspin_b200 import _lib
from hotspin_b200.sim import Batch, Simulation

pytestmark = pytest.mark.gpu

MU0 = 4e-7 * np.pi
MUB = 9.27400968202020202e-24
HSB_ERR_NONFINITE = 5


def _llg(**kw):
    ms = 8e5
    d = dict(size=(2, 16, 32), cellsize=(3e-9,) * 3, msat0T0=ms, lex=float(np.sqrt(2 * 1.3e-11 / (MU0 * ms * ms))),
             gamma_ll=2.211e5, alpha=(0.05,) * 3, b_ext=(0.0, 0.01, 0.02), demag=True, normalize=True)
    d.update(kw)
    return d


def _ttm(**kw):
    d = _llg(llb=True, normalize=False, tc=630.0, spin_j=0.5, n_spins=8e5 / (2 * MUB * 0.5), temperature=300.0,
             ttm=True, gamma_e=700.0, c_l=3e6, g_ep=6e17, k_e=90.0)
    d.update(kw)
    return d


def _m(size, seed=1, length=1.0):
    m = np.random.default_rng(seed).normal(size=(3,) + size)
    return length * m / np.sqrt((m * m).sum(0))


def _step_rc(sim, n):
    return sim._lib.hsb_sim_step(sim._h, int(n))


@pytest.mark.parametrize("solver", ["rk4", "heun", "dp45"])
def test_nan_in_m_reports_nonfinite(cuda, solver):
    kw = _llg()
    m = _m(kw["size"])
    m[1, 1, 3, 7] = np.nan
    with Simulation(**kw, solver=solver, dt=1e-15, rtol=1e-5, mindt=1e-20, maxdt=1e-12) as sim:
        sim.set("m", m)
        rc = _step_rc(sim, 5)
        assert rc == HSB_ERR_NONFINITE, (rc, sim._lib.hsb_last_error())
        st = sim.status()
        assert st["status"] & 1
        # the handle refuses to step until the state is replaced, then runs again
        assert _step_rc(sim, 1) == HSB_ERR_NONFINITE
        sim.set("m", _m(kw["size"]))
        sim.set_time(0.0, 1e-15)
        assert _step_rc(sim, 3) == 0, sim._lib.hsb_last_error()
        assert sim.status()["status"] == 0 and np.isfinite(sim.get("m")).all()


def test_inf_in_electron_temperature_reports_nonfinite(cuda):
    kw = _ttm()
    size = kw["size"]
    from oracle import fields as F
    Te = np.full(size, 300.0)
    Te[0, 5, 5] = np.inf
    with Simulation(**kw, solver="dp45", dt=1e-16, rtol=1e-5, mindt=1e-20, maxdt=1e-13) as sim:
        sim.set("m", _m(size, 2, F.equilibrium_m(300.0, 630.0, 0.5)))
        sim.set("Te", Te)
        sim.set("Tl", np.full(size, 300.0))
        rc = _step_rc(sim, 3)
        assert rc == HSB_ERR_NONFINITE, (rc, sim._lib.hsb_last_error())
        assert sim.status()["status"] & 1


def test_unreachable_tolerance_flags_floor_steps(cuda):
    kw = _llg()
    with Simulation(**kw, solver="dp45", dt=1e-15, rtol=1e-12, mindt=1e-15, maxdt=1e-15) as sim:
        sim.set("m", _m(kw["size"], 3))
        sim.step(4)                              # steps are taken at the floor
        st = sim.status()
    assert st["steps"] == 4 and st["rejects"] == 0
    assert st["err"] > 1.0
    assert st["status"] & 2 and not st["status"] & 1


def test_reachable_tolerance_sets_no_flag(cuda):
    kw = _llg()
    with Simulation(**kw, solver="dp45", dt=1e-15, rtol=1e-5, mindt=1e-20, maxdt=1e-12) as sim:
        sim.set("m", _m(kw["size"], 3))
        sim.step(10)
        assert sim.status()["status"] == 0


def _class():
    from hotspin_b200 import serve
    d = dict(size=(1, 32, 64), cellsize=(3e-9,) * 3, pbc=(0, 0, 0), msat0T0=8e5,
             lex=float(np.sqrt(2 * 1.3e-11 / (MU0 * 8e5 ** 2))), alpha=(0.05,) * 3, b_ext=(0.0, 0.01, 0.02),
             demag=True, normalize=True, temperature=0.0, thermal=True, seed=7, solver="dp45", dt=1e-15,
             rtol=1e-5, mindt=1e-22, maxdt=1e-12)
    return d, serve.class_desc(d)


def _run(release_mid):
    d, cls = _class()
    size = d["size"]
    out = {}
    with Batch(3, **cls) as b:
        for s in range(3):
            b.admit(s, _m(size, 10 + s), 1.5e-12, **dict(d, temperature=100.0 * s, seed=20 + s))
        released = False
        for _ in range(100000):
            b.launch(1)
            if release_mid and not released:
                b.release(1)                     # enqueued behind the running class graph
                released = True
            while not b.poll():
                pass
            if not any(b.slot_status(s)["active"] for s in (0, 2)):
                break
        for s in (0, 2):
            out[s] = (b.slot_get(s, "m"), b.slot_status(s))
        st1 = b.slot_status(1)
    return out, st1


def test_release_of_running_slot_leaves_others_bitwise(cuda):
    base, _ = _run(False)
    rel, st1 = _run(True)
    assert not st1["active"] and st1["t"] < 1.5e-12
    for s in (0, 2):
        np.testing.assert_array_equal(base[s][0], rel[s][0])
        assert base[s][1]["steps"] == rel[s][1]["steps"]


@pytest.mark.parametrize("thermal", [False, True])
def test_checkpoint_restore_repeats_bitwise(cuda, thermal):
    kw = _ttm(thermal=thermal, seed=5, laser_p0=5e20, laser_t0=5e-14, laser_fwhm=1e-13)
    size = kw["size"]
    from oracle import fields as F
    with Simulation(**kw, solver="dp45", dt=1e-16, rtol=1e-5, mindt=1e-20, maxdt=1e-13) as sim:
        sim.set("m", _m(size, 4, F.equilibrium_m(300.0, 630.0, 0.5)))
        sim.set("Te", np.full(size, 300.0))
        sim.set("Tl", np.full(size, 300.0))
        sim.step(3)
        sim.checkpoint()
        s0 = sim.status()
        sim.step(6)
        m1, T1, s1 = sim.get("m"), sim.get("Te"), sim.status()
        sim.restore()
        assert sim.status()["t"] == s0["t"] and sim.status()["steps"] == s0["steps"]
        sim.step(6)
        m2, T2, s2 = sim.get("m"), sim.get("Te"), sim.status()
    np.testing.assert_array_equal(m1, m2)
    np.testing.assert_array_equal(T1, T2)
    assert (s1["t"], s1["steps"], s1["attempts"]) == (s2["t"], s2["steps"], s2["attempts"])


def test_restore_without_checkpoint_is_refused(cuda):
    kw = _llg()
    with Simulation(**kw, solver="rk4", dt=1e-15) as sim:
        rc = sim._lib.hsb_sim_restore(sim._h)
        assert rc == 1 and b"checkpoint" in sim._lib.hsb_last_error()
