"""Accuracy of the FP32 device path against the FP64 oracle on reduced versions of the
benchmark workloads: max |dm| (and |dT| for the two-temperature model) and the relative
energy error after the stated integration.

The full-size workloads are too large for the FP64 host oracle; each case keeps the
workload's physics, integrator and tolerance on a grid the oracle integrates in seconds.
Thermal fields are off (their parity is trajectory-level and is covered by test_gpu_sim.py);
the thin-film LLG case's random start is replaced by the reference's smooth standard-problem
start (the random start is chaotic, so no implementation stays within 1e-5 of another on it).
The LLB cases' energy tolerance is looser than their |dm| one: the longitudinal-field energy
is as stiff in |m| as the longitudinal relaxation (the reason those solves need femtosecond
steps), so a |m| difference at FP32 rounding moves it by ~1e-4 of the total.
Run with `-s` to see the table.
"""
import numpy as np
import pytest

from hotspin_b200.sim import Simulation
from oracle import fields as F
from oracle.model import Model, Spec
from oracle.solvers import Integrator

pytestmark = pytest.mark.gpu

MUB = F.MUB


def _lex(ms, a):
    return float(np.sqrt(2 * a / (F.MU0 * ms * ms)))


def _tilted(size, deg, seed, length=1.0):
    rng = np.random.default_rng(seed)
    th = np.deg2rad(deg) * rng.random(size)
    ph = 2 * np.pi * rng.random(size)
    return length * np.stack([np.cos(th), np.sin(th) * np.sin(ph), np.sin(th) * np.cos(ph)])


def _random_unit(size, seed):
    m = np.random.default_rng(seed).normal(size=(3,) + size)
    return m / np.sqrt((m * m).sum(0))


CASES = {
    # thin-film plain LLG (128x32x1), RK4 50 fs (smooth start, 1000 steps)
    "llg_film_rk4": dict(
        kw=dict(size=(1, 32, 128), cellsize=(3e-9, 3.90625e-9, 3.90625e-9), msat0T0=8e5, lex=_lex(8e5, 1.3e-11),
                gamma_ll=F.GAMMA0 / (1 + 0.02 ** 2), alpha=(0.02,) * 3, b_ext=(0.0, 0.012, 0.016), demag=True,
                normalize=True),
        init=lambda size: {"m": np.stack([np.zeros(size), np.full(size, 2 ** -0.5), np.full(size, 2 ** -0.5)])},
        solver="rk4", dt=50e-15, steps=1000, tol_m=1e-5, tol_e=1e-5),
    # LLB at 300 K, FePt-like, uniaxial Ku along z (program X), DP45 1e-5
    "llb_fept_dp45": dict(
        kw=dict(size=(8, 16, 16), cellsize=(2e-9,) * 3, msat0T0=1.1e6, lex=_lex(1.1e6, 1e-11), gamma_ll=F.GAMMA0,
                alpha=(0.1,) * 3, ku=7e6, anis_u=(1.0, 0.0, 0.0), demag=True, llb=True, tc=700.0, spin_j=0.5,
                n_spins=1.1e6 / (2 * MUB * 0.5), temperature=300.0),
        init=lambda size: {"m": _tilted(size, 5.0, 2, F.equilibrium_m(300.0, 700.0, 0.5))},
        solver="dp45", dt=1e-16, t_end=1e-12, tol_m=1e-5, tol_e=5e-4),
    # two-temperature model + LLB with the laser pulse, DP45 1e-5
    "ttm_llb_laser_dp45": dict(
        kw=dict(size=(4, 32, 32), cellsize=(4e-9,) * 3, msat0T0=8e5, lex=_lex(8e5, 1.3e-11),
                gamma_ll=F.GAMMA0 / (1 + 0.02 ** 2), alpha=(0.02,) * 3, b_ext=(0.02, 0.0, 0.0), demag=True, llb=True,
                tc=630.0, spin_j=0.5, n_spins=8e5 / (2 * MUB * 0.5), temperature=300.0, ttm=True, gamma_e=700.0,
                c_l=3e6, g_ep=6e17, k_e=90.0, k_l=0.0, laser_p0=5e20, laser_t0=5e-14, laser_fwhm=1e-13,
                laser_sigma=40e-9),
        init=lambda size: dict(m=_tilted(size, 5.0, 3, F.equilibrium_m(300.0, 630.0, 0.5)),
                               Te=np.full(size, 300.0), Tl=np.full(size, 300.0)),
        solver="dp45", dt=2e-16, t_end=5e-13, tol_m=1e-5, tol_e=1e-5),
    # large-instance LLG physics on the multi-pass FFT path (L0 = 64), RK4 20 fs, alpha 0.5
    "llg_multipass_rk4": dict(
        kw=dict(size=(32, 16, 16), cellsize=(2e-9,) * 3, msat0T0=8e5, lex=_lex(8e5, 1.3e-11),
                gamma_ll=F.GAMMA0 / (1 + 0.5 ** 2), alpha=(0.5,) * 3, demag=True, normalize=True),
        init=lambda size: {"m": _random_unit(size, 5)},
        solver="rk4", dt=20e-15, steps=100, tol_m=1e-5, tol_e=1e-5),
}


@pytest.mark.parametrize("name", list(CASES))
def test_accuracy_against_oracle(cuda, name):
    case = CASES[name]
    kw = case["kw"]
    y0 = case["init"](kw["size"])
    spec = Spec(**kw)
    model = Model(spec)
    solver = case["solver"]
    if solver == "rk4":
        it = Integrator(model, y0, "rk4", case["dt"])
        it.run_steps(case["steps"])
    else:
        it = Integrator(model, y0, "dp45", case["dt"], rtol=1e-5, mindt=1e-20, maxdt=1e-12)
        it.run_until(case["t_end"])
    with Simulation(**kw, solver=solver, dt=case["dt"], rtol=1e-5, mindt=1e-20, maxdt=1e-12) as sim:
        for k, v in y0.items():
            sim.set(k, v)
        if solver == "rk4":
            sim.step(case["steps"])
        else:
            sim.run_until(case["t_end"])
        m = sim.get("m")
        E = sim.energy()
        st = sim.status()
        Te = sim.get("Te") if kw.get("ttm") else None
    dm = float(np.abs(m - it.y["m"]).max())
    Eo = model.energy(it.y)
    de = abs(E - Eo) / abs(Eo)
    extra = ""
    if Te is not None:
        dT = float(np.abs(Te - it.y["Te"]).max() / it.y["Te"].max())
        extra = " rel max|dTe| %.2e" % dT
        assert dT < 1e-5
    print("\n[accuracy] %-22s cells %7d steps %5d (oracle %5d)  max|dm| %.2e  rel dE %.2e%s"
          % (name, int(np.prod(kw["size"])), st["steps"], it.step_count, dm, de, extra))
    assert dm < case["tol_m"]
    assert de < case["tol_e"]
