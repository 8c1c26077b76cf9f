"""Stochastic runs checked statistically at 3 sigma, at several temperatures.

1. Same Philox stream: the device and the FP64 oracle (which restates the same Philox4x32-10
   stream per cell and step) integrate an ensemble of uncoupled macrospins with the Brown
   thermal field by fixed-step Heun; the ensemble mean and variance of m along the field agree
   within 3 sigma of their sampling errors (in practice far closer: the trajectories are the
   same up to FP32 rounding).
2. Boltzmann equilibrium: a large ensemble relaxed by the device to equilibrium has the
   Langevin mean <cos theta> = L(xi) = coth(xi) - 1/xi and variance 1 - 2 L(xi)/xi - L(xi)^2
   within 3 sigma, xi = Ms V B / (kB T_eff).  hotspin's noise (variance
   2 kB T lambda / (mu0 Ms V gamma_LL dt), mod_brown.go:125-145) drives the Landau-Lifshitz
   form of the LLBar equation, whose stationary temperature is T (1 + lambda^2) when gamma_LL
   is the bare gyromagnetic ratio: T_eff below.  Snapshots are three relaxation times apart
   (correlation below e^-3), so spins and snapshots are close to independent samples.  The
   same Heun scheme on macrospins in NumPy (65536 spins, lambda 0.1, 300 K) gives <cos theta>
   at 1.7 and 0.3 sigma from L(xi / (1 + lambda^2)) at dt = 2e-14 and 4e-14 s and 8 sigma away
   from L(xi): the T (1 + lambda^2) temperature is the scheme's, and its time-step bias is
   below the sampling error.
"""
import numpy as np
import pytest

from hotspin_b200.sim import Simulation
from oracle import fields as F
from oracle.model import Model, Spec
from oracle.solvers import Integrator

pytestmark = pytest.mark.gpu

MS, CS, LAM = 8e5, 3e-9, 0.1


def _kw(size, T, B, seed):
    return dict(size=size, cellsize=(CS,) * 3, msat0T0=MS, gamma_ll=F.GAMMA0, alpha=(LAM,) * 3, normalize=True,
                b_ext=(B, 0.0, 0.0), thermal=True, seed=seed, temperature=T)


def _moments(v):
    n = v.size
    mean = float(v.mean())
    var = float(v.var())
    mu4 = float(((v - mean) ** 4).mean())
    return mean, var, np.sqrt(var / n), np.sqrt(max(mu4 - var * var, 0.0) / n)


@pytest.mark.parametrize("T", [100.0, 300.0, 600.0])
def test_same_stream_ensemble_matches_oracle_3sigma(cuda, T):
    size, B, dt, nsteps = (1, 64, 64), 0.2, 2e-14, 200
    kw = _kw(size, T, B, seed=31)
    rng = np.random.default_rng(17)
    m0 = rng.normal(size=(3,) + size)
    m0 /= np.sqrt((m0 * m0).sum(0))
    it = Integrator(Model(Spec(**kw)), {"m": m0}, "heun", dt)
    it.run_steps(nsteps)
    with Simulation(**kw, solver="heun", dt=dt) as sim:
        sim.set("m", m0)
        sim.step(nsteps)
        m = sim.get("m")
    a = _moments(m[0].ravel())
    b = _moments(it.y["m"][0].ravel())
    print("\n[same stream T=%g] mean %.5f / %.5f  var %.5f / %.5f  max|dm| %.1e"
          % (T, a[0], b[0], a[1], b[1], np.abs(m - it.y["m"]).max()))
    assert abs(a[0] - b[0]) < 3 * np.hypot(a[2], b[2])
    assert abs(a[1] - b[1]) < 3 * np.hypot(a[3], b[3])


@pytest.mark.parametrize("T", [150.0, 600.0])
def test_dp45_same_stream_ensemble_matches_oracle_3sigma(cuda, T):
    """The adaptive DP45 path with the thermal field (the benchmark's integrator): step sizes
    follow FP32 vs FP64 error estimates, so trajectories separate at the noise scale, and the
    ensembles are compared statistically."""
    size, B = (1, 64, 64), 0.2
    kw = _kw(size, T, B, seed=41)
    rng = np.random.default_rng(19)
    m0 = rng.normal(size=(3,) + size)
    m0 /= np.sqrt((m0 * m0).sum(0))
    t_end = 5e-12
    it = Integrator(Model(Spec(**kw)), {"m": m0}, "dp45", 1e-15, rtol=1e-5, mindt=1e-20, maxdt=1e-12)
    it.run_until(t_end)
    with Simulation(**kw, solver="dp45", dt=1e-15, rtol=1e-5, mindt=1e-20, maxdt=1e-12) as sim:
        sim.set("m", m0)
        sim.run_until(t_end)
        m = sim.get("m")
    for c in range(3):
        a = _moments(m[c].ravel())
        b = _moments(it.y["m"][c].ravel())
        assert abs(a[0] - b[0]) < 3 * np.hypot(a[2], b[2]), (c, a, b)
        assert abs(a[1] - b[1]) < 3 * np.hypot(a[3], b[3]), (c, a, b)


@pytest.mark.late
@pytest.mark.parametrize("T", [150.0, 300.0, 600.0])
def test_equilibrium_is_boltzmann_3sigma(cuda, T):
    size, B, dt = (4, 128, 128), 0.383, 2e-14
    T_eff = T * (1 + LAM * LAM)
    xi = MS * CS ** 3 * B / (F.KB * T_eff)
    L = 1.0 / np.tanh(xi) - 1.0 / xi
    var_L = 1.0 - 2.0 * L / xi - L * L
    tau = 1.0 / (LAM * F.GAMMA0 * B)               # relaxation time
    kw = _kw(size, T, B, seed=int(T))
    samples = []
    with Simulation(**kw, solver="heun", dt=dt) as sim:
        m = np.zeros((3,) + size)
        m[0] = 1.0
        sim.set("m", m)
        per = int(round(3 * tau / dt))
        sim.step(3 * per)                           # nine relaxation times to equilibrium
        for _ in range(10):
            sim.step(per)
            samples.append(sim.get("m")[0].ravel())
    v = np.concatenate(samples)
    mean, var, s_mean, s_var = _moments(v)
    print("\n[Boltzmann T=%g xi=%.3f] <m0> %.5f (L %.5f, 3 sigma %.1e)  var %.5f (%.5f, 3 sigma %.1e)"
          % (T, xi, mean, L, 3 * s_mean, var, var_L, 3 * s_var))
    assert abs(mean - L) < 3 * s_mean
    assert abs(var - var_L) < 3 * s_var
