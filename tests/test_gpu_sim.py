"""Fused FP32 right-hand side and integrators (simulation handle) against the FP64 oracle."""
import numpy as np
import pytest

from hotspin_b200.sim import Simulation
from oracle import fields as F
from oracle.model import Model, Spec
from oracle.solvers import Integrator
from tests.gpu_util import rel_err

pytestmark = pytest.mark.gpu

MS, AEX = 8e5, 1.3e-11
LEX = float(np.sqrt(2 * AEX / (F.MU0 * MS * MS)))


def unit(seed, size):
    m = np.random.default_rng(seed).normal(size=(3,) + size)
    return m / np.sqrt((m * m).sum(0))


def pair(**kw):
    """The same problem as an oracle Spec and a device Simulation."""
    spec = Spec(**kw)
    desc = dict(kw)
    desc.pop("msat_mask", None)
    desc.pop("lex_mask", None)
    return spec, desc


LLG = dict(size=(2, 16, 32), cellsize=(3e-9, 3.9e-9, 3.9e-9), msat0T0=MS, lex=LEX,
           gamma_ll=F.GAMMA0 / (1 + 0.02 ** 2), alpha=(0.02, 0.02, 0.02), b_ext=(0.0, 0.012, 0.016),
           demag=True, normalize=True, ku=2e4, anis_u=(0.3, 0.0, 1.0))
LLB = dict(size=(4, 16, 16), cellsize=(2e-9, 2e-9, 2e-9), msat0T0=1.1e6, lex=float(np.sqrt(2 * 1e-11 / (F.MU0 * 1.1e6 ** 2))),
           gamma_ll=F.GAMMA0, alpha=(0.1, 0.1, 0.1), ku=7e6, anis_u=(1.0, 0.0, 0.0), demag=True, llb=True,
           tc=700.0, spin_j=0.5, n_spins=1.1e6 / (2 * F.MUB * 0.5), temperature=300.0)
TTM = dict(LLB, size=(2, 16, 32), cellsize=(4e-9, 4e-9, 4e-9), msat0T0=MS, lex=LEX, tc=630.0,
           n_spins=MS / (2 * F.MUB * 0.5), alpha=(0.02, 0.02, 0.02), ku=0.0, ttm=True, gamma_e=700.0, c_l=3e6,
           g_ep=6e17, k_e=90.0, k_l=0.0, laser_p0=5e20, laser_t0=0.0, laser_fwhm=1e-13, laser_sigma=40e-9)


def state(kw, seed=5):
    size = kw["size"]
    m = unit(seed, size)
    y = {}
    if kw.get("llb"):
        m = m * np.random.default_rng(seed + 1).uniform(0.6, 0.95, size=size)
    y["m"] = m
    if kw.get("ttm"):
        rng = np.random.default_rng(seed + 2)
        y["Te"] = rng.uniform(300.0, 900.0, size=size)
        y["Tl"] = rng.uniform(300.0, 400.0, size=size)
    return y


@pytest.mark.parametrize("kw", [LLG, LLB, TTM], ids=["llg", "llb", "ttm"])
@pytest.mark.parametrize("thermal", [False, True])
def test_rhs_matches_oracle(cuda, kw, thermal):
    kw = dict(kw, thermal=thermal, seed=77, dt=1e-14, solver="rk4")
    if thermal and not kw.get("llb"):
        kw["temperature"] = 200.0
    spec, desc = pair(**{k: v for k, v in kw.items() if k not in ("solver", "dt")})
    y = state(kw)
    model = Model(spec)
    model.set_thermal(0, kw["dt"], model.spin_temperature(y))
    want = model.rhs(0.0, y)
    with Simulation(**desc, solver="rk4", dt=kw["dt"]) as sim:
        for name, v in y.items():
            sim.set(name, v)
        k = sim.get("k")
    assert rel_err(k[:3], want["m"]) < 3e-5
    if kw.get("ttm"):
        assert rel_err(k[3], want["Te"]) < 3e-5
        assert rel_err(k[4], want["Tl"]) < 3e-5


@pytest.mark.parametrize("kw", [LLG, LLB, TTM], ids=["llg", "llb", "ttm"])
def test_max_torque_matches_oracle(cuda, kw):
    """hsb_sim_max_torque = max over cells of |gamma (m x H_eff)| of the oracle's field; twice in
    a row (the reduction word is cleared per call), and the state is untouched."""
    kw = dict(kw, thermal=False, dt=1e-14, solver="rk4")
    spec, desc = pair(**{k: v for k, v in kw.items() if k not in ("solver", "dt")})
    y = state(kw)
    model = Model(spec)
    m = F.normalize(y["m"]) if spec.normalize else y["m"]
    H = model.heff(dict(y, m=m))
    tau = F.llbar_torque(m, H, None, spec.gamma_ll)
    want = float(np.sqrt((tau * tau).sum(0)).max())
    with Simulation(**desc, solver="rk4", dt=kw["dt"]) as sim:
        for name, v in y.items():
            sim.set(name, v)
        got = [sim.max_torque(), sim.max_torque()]
        m_after = sim.get("m")
    assert got[0] == got[1]
    assert abs(got[0] - want) < 3e-5 * want
    assert np.abs(m_after - m).max() < 1e-6


def test_masks_rhs(cuda):
    size = (2, 8, 16)
    rng = np.random.default_rng(4)
    ms = rng.uniform(0.3, 1.0, size=size)
    ms[0, 3:5, 3:6] = 0.0
    lex = 1.0 / np.maximum(ms, 0.3)
    kw = dict(LLG, size=size)
    spec = Spec(**kw, msat_mask=ms, lex_mask=lex)
    y = state(kw)
    want = Model(spec).rhs(0.0, y)
    with Simulation(**kw, solver="rk4", dt=1e-14) as sim:
        sim.set("msat_mask", ms)
        sim.set("lex_mask", lex)
        sim.set("m", y["m"])
        k = sim.get("k")
        assert rel_err(k, want["m"]) < 3e-5
        assert np.all(k[:, 0, 3:5, 3:6] == 0.0)
        E = sim.energy()
    assert abs(E - Model(spec).energy(y)) < 1e-4 * abs(Model(spec).energy(y))


@pytest.mark.parametrize("size", [(3, 5, 7), (2, 6, 12)])
def test_rhs_without_demag_any_size(cuda, size):
    """Sizes with no power-of-two padding run without demag; N2 % 4 != 0 takes the
    one-cell-per-thread kernel, N2 % 4 == 0 the four-cell one."""
    kw = dict(TTM, size=size, demag=False, laser_sigma=10e-9)
    spec, desc = pair(**kw)
    y = state(kw)
    want = Model(spec).rhs(0.0, y)
    with Simulation(**desc, solver="rk4", dt=1e-15) as sim:
        for name, v in y.items():
            sim.set(name, v)
        k = sim.get("k")
    assert rel_err(k[:3], want["m"]) < 3e-5
    assert rel_err(k[3], want["Te"]) < 3e-5


@pytest.mark.parametrize("method", ["euler", "heun", "rk4"])
def test_fixed_step_trajectory(cuda, method):
    kw = dict(LLG)
    spec, desc = pair(**kw)
    y = state(kw, seed=9)
    it = Integrator(Model(spec), y, method, 2e-14)
    it.run_steps(25)
    with Simulation(**desc, solver=method, dt=2e-14) as sim:
        sim.set("m", y["m"])
        sim.step(25)
        st = sim.status()
        m = sim.get("m")
    assert st["steps"] == 25 and st["t"] == pytest.approx(25 * 2e-14, rel=1e-12)
    assert np.abs(m - it.y["m"]).max() < 1e-5


def test_rk4_smooth_4000_steps_parity(cuda):
    """Well-conditioned thin film (uniform start, the reference's stdproblem4 geometry):
    4000 RK4 steps of 50 fs stay within 1e-5 max|dm| of the FP64 oracle."""
    size = (1, 32, 128)
    kw = dict(size=size, cellsize=(3e-9, 500e-9 / 128, 125e-9 / 32), msat0T0=MS, lex=LEX,
              gamma_ll=F.GAMMA0 / (1 + 0.02 ** 2), alpha=(0.02,) * 3, b_ext=(0.0, 4.3e-3, -24.6e-3),
              demag=True, normalize=True)
    spec, desc = pair(**kw)
    m0 = np.zeros((3,) + size)
    m0[1] = m0[2] = 1 / np.sqrt(2)
    it = Integrator(Model(spec), {"m": m0}, "rk4", 50e-15)
    it.run_steps(4000)
    with Simulation(**desc, solver="rk4", dt=50e-15) as sim:
        sim.set("m", m0)
        sim.step(4000)
        m = sim.get("m")
        E = sim.energy()
    assert np.abs(m - it.y["m"]).max() < 1e-5
    Eo = Model(spec).energy(it.y)
    assert abs(E - Eo) < 1e-5 * abs(Eo)


@pytest.mark.parametrize("kw", [LLG, TTM], ids=["llg", "ttm"])
def test_dp45_matches_oracle(cuda, kw):
    kw = dict(kw, thermal=False)
    spec, desc = pair(**kw)
    y = state(kw, seed=11)
    it = Integrator(Model(spec), y, "dp45", 1e-15, rtol=1e-5, mindt=1e-20, maxdt=1e-12)
    t_end = 2e-13
    it.run_until(t_end)
    with Simulation(**desc, solver="dp45", dt=1e-15, rtol=1e-5, mindt=1e-20, maxdt=1e-12) as sim:
        for name, v in y.items():
            sim.set(name, v)
        sim.run_until(t_end)
        st = sim.status()
        m = sim.get("m")
        T = sim.get("Te") if kw.get("ttm") else None
    assert st["t"] == pytest.approx(t_end, rel=1e-9)
    assert abs(st["steps"] - it.step_count) <= max(2, it.step_count // 10)
    assert np.abs(m - it.y["m"]).max() < 1e-5
    if T is not None:
        assert rel_err(T, it.y["Te"]) < 1e-5


def test_thermal_field_statistics(cuda):
    """Single uncoupled spins at finite T: the thermal field has zero mean and the variance
    2 kB T lambda / (mu0 Ms V gamma dt) per component (mod_brown.go:125-145)."""
    size = (4, 64, 64)
    kw = dict(size=size, cellsize=(2e-9,) * 3, msat0T0=MS, gamma_ll=F.GAMMA0, alpha=(0.1, 0.1, 0.1),
              thermal=True, seed=2, temperature=300.0, solver="rk4", dt=1e-14)
    with Simulation(**kw) as sim:
        m = np.zeros((3,) + size)
        m[2] = 1.0
        sim.set("m", m)
        k = sim.get("k")
    # k = gamma (H x m) + gamma lambda H with m = z: k_x = gamma (H_y + lambda H_x) ...
    g = F.GAMMA0
    Hz = k[2] / (g * 0.1)
    var = F.thermal_prefactor(300.0, (2e-9,) * 3, g, 1e-14, 0.0, MS) * 0.1
    n = Hz.size
    assert abs(Hz.mean()) < 4 * np.sqrt(var / n)
    assert abs(Hz.var() / var - 1) < 4 * np.sqrt(2.0 / n)


@pytest.mark.parametrize("variant", [0, 1, 4])
def test_stage_kernel_variants_agree(cuda, variant):
    """Every stage-kernel variant integrates the same trajectories as the default one, up to
    FP32 rounding order: DP45 on TTM + LLB + demag + laser from a state near equilibrium, and
    fixed-step RK4 with the thermal field.  (Stochastic DP45 runs are compared statistically
    only: the noise amplitude scales with the accepted dt, and FP32 rounding in the error
    estimate moves the step sizes.)"""
    from hotspin_b200 import _lib
    lib = _lib.load()
    kw = dict(TTM, size=(2, 16, 32), seed=5, laser_t0=5e-14)
    size = kw["size"]
    rng = np.random.default_rng(12)
    th, ph = np.deg2rad(5.0) * rng.random(size), 2 * np.pi * rng.random(size)
    me = F.equilibrium_m(300.0, kw["tc"], 0.5)
    y = {"m": me * np.stack([np.cos(th), np.sin(th) * np.sin(ph), np.sin(th) * np.cos(ph)]),
         "Te": np.full(size, 300.0), "Tl": np.full(size, 300.0)}
    runs = [dict(thermal=False, solver="dp45", dt=1e-16, t_end=2e-13),
            dict(thermal=True, solver="rk4", dt=1e-15, steps=20)]
    default = lib.hsb_set_stage_variant(2)
    assert default == -1     # no variant forced outside this test
    try:
        for run in runs:
            out = {}
            for v in (2, variant):
                lib.hsb_set_stage_variant(v)
                with Simulation(**dict(kw, thermal=run["thermal"]), solver=run["solver"], dt=run["dt"], rtol=1e-5,
                                mindt=1e-20, maxdt=1e-13) as sim:
                    for name, val in y.items():
                        sim.set(name, val)
                    if "steps" in run:
                        sim.step(run["steps"])
                    else:
                        sim.run_until(run["t_end"])
                    out[v] = (sim.get("m"), sim.get("Te"), sim.status())
            (m2, T2, s2), (mv, Tv, sv) = out[2], out[variant]
            assert s2["t"] == pytest.approx(sv["t"], rel=1e-12)
            assert np.abs(m2 - mv).max() < 1e-5, run
            assert np.abs(T2 - Tv).max() < 1e-5 * T2.max(), run
    finally:
        lib.hsb_set_stage_variant(default)


def test_stage_tuning_picks_a_variant(cuda):
    """Each handle runs the stage-kernel variant its creation-time tuning picked."""
    from hotspin_b200 import _lib
    lib = _lib.load()
    with Simulation(**dict(LLG, size=(2, 16, 32)), solver="dp45", dt=1e-15) as sim:
        assert lib.hsb_stage_variant_of(sim._h) in (1, 2, 4)


def test_dump_of_a_simulation(cuda, tmp_path):
    """hotspin_b200.dump.write_simulation writes the handle's m and time as a #dump002 frame."""
    from hotspin_b200 import dump
    kw = dict(LLG, thermal=False)
    spec, desc = pair(**kw)
    y = state(kw)
    p = str(tmp_path / "m.dump")
    with Simulation(**desc, solver="rk4", dt=1e-14) as sim:
        sim.set("m", y["m"])
        sim.step(3)
        dump.write_simulation(p, sim)
        m = sim.get("m")
        t = sim.status()["t"]
    (data, hdr), = dump.read(p)
    assert np.array_equal(data, m.astype(np.float32))
    assert hdr["time"] == t and hdr["label"] == "m" and hdr["mesh"] == kw["size"]


def test_pointwise_laser_profile(cuda):
    """A (time, factor) laser table is interpolated linearly as hotspin's pointwise quantities
    are, zero outside its range: the two-temperature RHS matches the oracle's at times on a
    ramp, on a knot and past the table, and DP45 through the pulse matches the oracle's run.
    Batches refuse such tables."""
    from hotspin_b200 import _lib
    from hotspin_b200.sim import Batch
    tab = [(0.0, 0.0), (5e-14, 1.0), (1.2e-13, 0.3), (2.0e-13, 0.0)]
    kw = dict(TTM, thermal=False, laser_table=tab)
    spec, desc = pair(**kw)
    y = state(kw, seed=13)
    model = Model(spec)
    with Simulation(**desc, solver="rk4", dt=1e-15) as sim:
        for name, v in y.items():
            sim.set(name, v)
        for t in (2.5e-14, 5e-14, 9e-14, 2.5e-13):
            sim.set_time(t)
            k = sim.get("k")
            want = model.rhs(t, y)
            assert rel_err(k[3], want["Te"]) < 3e-5, t
            assert rel_err(k[:3], want["m"]) < 3e-5, t
    it = Integrator(Model(spec), y, "dp45", 1e-15, rtol=1e-5, mindt=1e-20, maxdt=1e-12)
    it.run_until(2e-13)
    with Simulation(**desc, solver="dp45", dt=1e-15, rtol=1e-5, mindt=1e-20, maxdt=1e-12) as sim:
        for name, v in y.items():
            sim.set(name, v)
        sim.run_until(2e-13)
        m, T = sim.get("m"), sim.get("Te")
    assert np.abs(m - it.y["m"]).max() < 1e-5
    assert rel_err(T, it.y["Te"]) < 1e-5
    with pytest.raises(_lib.HsbError, match="batches"):
        Batch(2, **dict(desc, size=(2, 16, 32)), solver="dp45", dt=1e-15)


def test_pointwise_applied_field(cuda):
    """A (t, Bx, By, Bz) table replaces the constant applied field, interpolated linearly at
    each stage's time and zero outside its range: the RHS and the energy match the oracle's at
    times on a ramp, on a knot and past the table, and RK4 across the ramps matches the
    oracle's steps."""
    from hotspin_b200 import _lib
    from hotspin_b200.sim import Batch
    tab = [(0.0, 0.0, 0.0, 0.0), (1e-12, 0.05, 0.0, 0.02), (2e-12, -0.05, 0.01, 0.0)]
    kw = dict(LLG, thermal=False, bext_table=tab)
    spec, desc = pair(**kw)
    y = state(kw, seed=17)
    model = Model(spec)
    with Simulation(**desc, solver="rk4", dt=1e-14) as sim:
        sim.set("m", y["m"])
        for t in (0.5e-12, 1e-12, 1.7e-12, 3e-12):
            sim.set_time(t)
            k = sim.get("k")
            assert rel_err(k[:3], model.rhs(t, y)["m"]) < 3e-5, t
            E, Eo = sim.energy(), model.energy(y, t)
            assert abs(E - Eo) < 1e-5 * abs(Eo), t
    it = Integrator(Model(spec), y, "rk4", 2e-14)
    it.run_steps(100)                      # 0 .. 2 ps: both ramps
    with Simulation(**desc, solver="rk4", dt=2e-14) as sim:
        sim.set("m", y["m"])
        sim.step(100)
        m = sim.get("m")
    assert np.abs(m - it.y["m"]).max() < 1e-5
    with pytest.raises(_lib.HsbError, match="batches"):
        Batch(2, **dict(desc, size=(2, 16, 32)), solver="dp45", dt=1e-15)


@pytest.mark.parametrize("kw", [LLG, LLB], ids=["llg", "llb"])
def test_second_order_relaxation_terms(cuda, kw):
    """llbar/damping/nonconservative/02/local and conservative/02/local on the handle (the
    generic stage kernel runs them): right-hand side and 20 RK4 steps against the oracle."""
    kw = dict(kw, thermal=False, mu_par=(0.02, 0.015, 0.01), mu_perp=(0.005, 0.01, 0.02))
    spec, desc = pair(**kw)
    y = state(kw, seed=23)
    want = Model(spec).rhs(0.0, y)
    it = Integrator(Model(spec), y, "rk4", 1e-14)
    it.run_steps(20)
    with Simulation(**desc, solver="rk4", dt=1e-14) as sim:
        sim.set("m", y["m"])
        k = sim.get("k")
        sim.step(20)
        m = sim.get("m")
    assert rel_err(k[:3], want["m"]) < 3e-5
    assert np.abs(m - it.y["m"]).max() < 1e-5


@pytest.mark.parametrize("pbc", [(0, 0, 0), (0, 2, 3)])
def test_nonlocal_relaxation_term(cuda, pbc):
    """llbar/damping/nonconservative/00/nonlocal on the handle (two passes of the generic stage
    kernel: effective fields stored, then their Laplacian): right-hand side and 20 RK4 steps
    against the oracle's restatement of llbar-nonlocal00nc.cu."""
    kw = dict(LLG, pbc=pbc, thermal=False, alpha_e=(2e-19, 3e-19, 1e-19))
    spec, desc = pair(**kw)
    y = state(kw, seed=29)
    want = Model(spec).rhs(0.0, y)
    it = Integrator(Model(spec), y, "rk4", 1e-14)
    it.run_steps(20)
    with Simulation(**desc, solver="rk4", dt=1e-14) as sim:
        sim.set("m", y["m"])
        k = sim.get("k")
        sim.step(20)
        m = sim.get("m")
    assert rel_err(k[:3], want["m"]) < 3e-5
    assert np.abs(m - it.y["m"]).max() < 1e-5
