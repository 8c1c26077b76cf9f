"""The device step-control rules, compiled for the host, against the oracle's restatement of
hotspin's solvers (no GPU needed).

``tests/native/rule_check.cu`` includes the same inline rule the rk12 controller kernel runs
(``hsb_rk12_rule`` in ``hsb_llg.cuh``); it is built here with nvcc as host code and driven
through ctypes on random and boundary error sequences.
"""
import ctypes
import math
import numpy as np
import pytest

from oracle.solvers import rk12_rule

@pytest.fixture(scope="module")
def rules(host_rules):
    lib = host_rules
    lib.rk12_rule_host.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                   ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.rk12_rule_host.restype = None
    return lib


def _device_rk12(lib, dt, mindt, maxdt, tries, errs, limits, nonfinite=False):
    e = (ctypes.c_float * 3)(*(list(errs) + [0.0] * (3 - len(errs))))
    m = (ctypes.c_double * 3)(*(list(limits) + [math.inf] * (3 - len(limits))))
    out = (ctypes.c_double * 6)()
    lib.rk12_rule_host(dt, mindt, maxdt, tries, e, m, len(errs), int(nonfinite), out)
    return dict(dt=out[0], accepted=bool(out[1]), status=int(out[2]), tries=int(out[3]), active=bool(out[4]),
                err=out[5])


def test_rk12_rule_matches_oracle_on_random_errors(rules):
    rng = np.random.default_rng(12)
    for _ in range(4000):
        neq = int(rng.integers(1, 4))
        limits = [float(10 ** rng.uniform(-6, -2)) for _ in range(neq)]
        if neq > 1 and rng.random() < 0.3:
            limits[int(rng.integers(1, neq))] = math.inf          # an uncontrolled temperature
        errs = [float(np.float32(lim * 10 ** rng.uniform(-3, 2))) if math.isfinite(lim)
                else float(np.float32(10 ** rng.uniform(-8, 0))) for lim in limits]
        if rng.random() < 0.05:
            errs[int(rng.integers(0, neq))] = 0.0
        dt = float(10 ** rng.uniform(-16, -12))
        mindt, maxdt = 1e-17, 1e-12
        acc, bad, ndt, emax = rk12_rule(dt, errs, limits, mindt, maxdt)
        got = _device_rk12(rules, dt, mindt, maxdt, 0, errs, limits)
        assert got["accepted"] == acc, (errs, limits, dt)
        assert got["dt"] == pytest.approx(ndt, rel=1e-14), (errs, limits, dt)
        assert got["err"] == pytest.approx(emax, rel=1e-12)
        assert got["status"] == (2 if (acc and bad) else 0)


def test_rk12_rule_order_of_equations(rules):
    """A bad equation makes the later ones take the cube-root factor (solve_rk12.go:170-183):
    with m good and Te bad the factor of m is a square root, with m bad and Te good the factor
    of Te is a cube root."""
    lim = [1e-4, 1e-2]
    for errs in ([1e-6, 5e-2], [5e-4, 1e-5], [1e-6, 1e-4]):
        acc, bad, ndt, _ = rk12_rule(1e-14, errs, lim, 1e-20, 1e-10)
        got = _device_rk12(rules, 1e-14, 1e-20, 1e-10, 0, errs, lim)
        assert got["accepted"] == acc and got["dt"] == pytest.approx(ndt, rel=1e-14)
    # m bad (ratio 0.2 -> cube root 0.585 x 0.8 = 0.468), Te far below its limit (would be 1.5)
    got = _device_rk12(rules, 1e-14, 1e-20, 1e-10, 0, [5e-4, 1e-8], lim)
    assert not got["accepted"] and got["dt"] == pytest.approx(1e-14 * 0.8 * 0.2 ** (1 / 3), rel=1e-12)


def test_rk12_rule_floor_and_retry_limit(rules):
    # bad, but dt_new clamps to mindt: kept, flagged (status 2)
    got = _device_rk12(rules, 1e-17, 1e-17, 1e-12, 0, [1.0], [1e-5])
    assert got["accepted"] and got["status"] == 2 and got["dt"] == 1e-17
    # the 12th bad attempt of a step stops the run (status 4), as the reference panics
    got = _device_rk12(rules, 1e-14, 1e-20, 1e-12, 10, [1.0], [1e-5])
    assert not got["accepted"] and got["active"] and got["tries"] == 11
    got = _device_rk12(rules, 1e-14, 1e-20, 1e-12, 11, [1.0], [1e-5])
    assert not got["accepted"] and not got["active"] and got["status"] == 4
    # a good step resets the retry count
    got = _device_rk12(rules, 1e-14, 1e-20, 1e-12, 7, [1e-7], [1e-5])
    assert got["accepted"] and got["tries"] == 0 and got["dt"] == pytest.approx(1.5e-14)


def test_rk12_rule_nonfinite(rules):
    got = _device_rk12(rules, 1e-14, 1e-20, 1e-12, 0, [float("nan")], [1e-5])
    assert not got["accepted"] and got["dt"] == pytest.approx(1e-15) and got["status"] == 0
    got = _device_rk12(rules, 1e-20, 1e-20, 1e-12, 0, [1e-6], [1e-5], nonfinite=True)
    assert not got["accepted"] and got["status"] & 1 and not got["active"]


def test_rk12_oracle_run_keeps_the_reference_retry_count():
    """The oracle's rk12 raises on the 12th bad attempt of a step, as solve_rk12.go:202-204."""
    from oracle.model import Model, Spec
    from oracle.solvers import Integrator
    ms = 8e5
    kw = dict(size=(1, 4, 4), cellsize=(3e-9,) * 3, msat0T0=ms, lex=float(np.sqrt(2 * 1.3e-11 / (4e-7 * np.pi * ms * ms))),
              gamma_ll=2.211e5, alpha=(0.1,) * 3, b_ext=(0.0, 0.0, 1.0), normalize=True)
    m = np.random.default_rng(1).normal(size=(3, 1, 4, 4))
    it = Integrator(Model(Spec(**kw)), {"m": m}, "rk12", 1e-11, mindt=1e-30, maxdt=1e-9, maxerr=1e-30)
    with pytest.raises(RuntimeError, match="cannot converge"):
        it.step()
    assert it.bad_steps == 11


def _dp45_host(lib):
    f = lib.dp45_rule_host
    f.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_int]
    f.restype = None
    return f


def test_dp45_rule_matches_oracle_controller(rules):
    """hsb_dp45_rule (the device's DP45 controller) against the oracle's _dp45 step control on
    random, boundary and non-finite errors: accept / reject, the next dt, the counters, the
    t_stop clamp and the status bits."""
    f = _dp45_host(rules)
    rng = np.random.default_rng(11)
    errs = list(np.exp(rng.uniform(np.log(1e-12), np.log(1e6), 400))) + [0.0, 1.0, np.nextafter(1.0, 2.0), 1e-30,
                                                                        3.0e38, float("inf"), float("nan")]
    for k, e in enumerate(errs):
        e32 = float(np.float32(e))
        dt = float(np.exp(rng.uniform(np.log(1e-18), np.log(1e-12))))
        mindt = dt if k % 7 == 0 else 1e-22          # every 7th attempt at the floor
        maxdt = float(dt * rng.uniform(0.5, 20.0))
        t0 = float(rng.uniform(0.0, 1e-11))
        t_stop = t0 + dt * float(rng.choice([0.5, 1.0, 1.3, 3.0, 100.0])) if k % 3 == 0 else 0.0
        sd = HostWord(rules, t=t0, dt=dt, mindt=mindt, maxdt=maxdt, t_stop=t_stop, step_stop=-1, active=1)
        f(sd.p, e32, 0)
        # the oracle's rule (oracle/solvers.py _dp45) and the device's t_stop / status handling
        finite = np.isfinite(e32)
        accept = finite and (e32 <= 1.0 or dt <= mindt)
        fac = 0.2 if not finite else (5.0 if e32 == 0.0 else 0.9 * e32 ** -0.2)
        fac = min(max(fac, 0.2), 5.0 if accept else 1.0)
        nd = min(max(dt * fac, mindt), maxdt)
        t1 = t0 + dt if accept else t0
        active = 1
        if t_stop > 0.0:
            rem = t_stop - t1
            if rem <= 1e-6 * nd or rem <= 0.0:
                active = 0
            elif nd > rem:
                nd = rem
        floor = dt <= mindt
        status = (1 if floor and not finite else 0) | (2 if floor and (not accept or e32 > 1.0) else 0)
        if status & 1:
            active = 0
        assert sd["step"] == (1 if accept else 0), (e32, dt, mindt)
        assert sd["rejects"] == (0 if accept else 1)
        assert sd["cur"] == (1 if accept else 0) and sd["kslot"] == (1 if accept else 0)
        assert sd["t"] == t1
        assert sd["dt"] == pytest.approx(nd, rel=1e-14)
        assert sd["active"] == active
        assert int(sd["status"]) == status, (e32, dt, mindt, int(sd["status"]), status)
        if finite:
            assert sd["err"] == e32
        sd.close()
    # the non-finite flag of the attempt rejects whatever the error says
    sd = HostWord(rules, t=0.0, dt=1e-15, mindt=1e-22, maxdt=1e-12, step_stop=-1, active=1)
    f(sd.p, 0.5, 1)
    assert sd["step"] == 0 and sd["dt"] == pytest.approx(2e-16, rel=1e-14) and int(sd["status"]) == 0
    sd.close()


# ---------------------------------------------------------------- implicit solvers, emulated
# The device runs am12 / bdf-euler as a fixed sequence of gated launches (hsb_sim.cu
# enqueue_attempt): sweeps (k_imp_sweep) fold per-channel maxima into the solver word and the
# decision kernel (hsb_imp_rule, built here for the host) acts on it.  These tests replay that
# launch sequence in FP64 with the oracle's right-hand side and the host-built rules, and check
# that it takes the same steps as the oracle's restatement of the reference solvers.

AM_PRED, AM_CORR, AM_ERR, BDF_EULER, BDF_SWEEP, AM_EULER = range(6)
R_AM_BEGIN, R_AM_ITER_PRED, R_AM_ITER_CORR, R_AM_PRED_END, R_AM_CORR_END, R_AM_FINAL, R_BDF_BEGIN, R_BDF_ITER, \
    R_BDF_CLEAR = range(9)
CHANNELS = {"m": (0, 3), "Te": (3, 1), "Tl": (4, 1)}


class HostWord:
    """A device solver word (HsbSolverDev) in host memory, driven by the host build of the rules."""

    def __init__(self, lib, **fields):
        for name, res, args in (("hsd_new", ctypes.c_void_p, []), ("hsd_free", None, [ctypes.c_void_p]),
                                ("hsd_get", ctypes.c_double, [ctypes.c_void_p, ctypes.c_char_p]),
                                ("hsd_set", None, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_double]),
                                ("hsd_fold", None, [ctypes.c_void_p, ctypes.c_int, ctypes.c_float]),
                                ("imp_rule_host", None, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                                         ctypes.POINTER(ctypes.c_double), ctypes.c_double,
                                                         ctypes.c_int, ctypes.c_int, ctypes.c_int])):
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        self.lib = lib
        self.p = lib.hsd_new()
        for k, v in fields.items():
            self[k] = v

    def __getitem__(self, k):
        return self.lib.hsd_get(self.p, k.encode())

    def __setitem__(self, k, v):
        self.lib.hsd_set(self.p, k.encode(), float(v))

    def fold(self, c, v):
        self.lib.hsd_fold(self.p, c, float(v))

    def rule(self, which, abs_err=(1e-4,) * 3, rel_err=(1e-3,) * 3, max_iter_err=1e-5, max_iter=3, neq=1, eq=0):
        a = (ctypes.c_double * 3)(*abs_err)
        r = (ctypes.c_double * 3)(*rel_err)
        self.lib.imp_rule_host(self.p, which, a, r, max_iter_err, max_iter, neq, eq)

    def close(self):
        self.lib.hsd_free(self.p)


def _fix(y, normalize):
    from oracle import fields as F
    if normalize:
        y = dict(y)
        y["m"] = F.normalize(y["m"])
    return y


def _chan(key, arr):
    """(channel index, array) pairs of an equation's array."""
    c0, nc = CHANNELS[key]
    return [(c0 + j, arr[j] if nc == 3 else arr) for j in range(nc)]


def emulate_am12(lib, model, y0, dt, nsteps, mindt, maxdt, abs_err, rel_err):
    """enqueue_attempt's SOLVER_AM12 sequence, attempt after attempt, until nsteps steps."""
    f, norm = model.rhs, model.s.normalize
    keys = [k for k in ("m", "Te", "Tl") if k in y0]
    neq = len(keys)
    ab = [abs_err[k] for k in keys] + [1.0] * (3 - neq)
    rl = [rel_err[k] for k in keys] + [1.0] * (3 - neq)
    sd = HostWord(lib, dt=dt, mindt=mindt, maxdt=maxdt, step_stop=nsteps)
    Y = {k: np.array(v, dtype=np.float64) for k, v in y0.items()}
    R = lambda which: sd.rule(which, ab, rl, neq=neq)
    trace = []
    while sd["active"]:
        t0, h = sd["t"], sd["dt"]
        R(R_AM_BEGIN)
        k0 = f(t0, Y)
        W = _fix({k: Y[k] + h * k0[k] for k in keys}, norm)
        k1 = f(t0 + h, W)
        k2 = None
        up = uc = None
        for phase in (0, 1):
            for j in range(6):
                if sd["active"] and sd["it_active"]:
                    h = sd["dt"]
                    dy = k2 if sd["dysel"] else k1
                    if phase == 0:
                        new = {k: Y[k] + h * dy[k] for k in keys}
                        prev = W
                    else:
                        new = {k: Y[k] + 0.5 * h * (dy[k] + k0[k]) for k in keys}
                        prev = up if sd["prevsel"] else W
                    for k in keys:
                        for (c, a), (_, b) in zip(_chan(k, prev[k]), _chan(k, new[k])):
                            sd.fold(c, np.abs(a - b).max())
                            sd.fold(5 + c, np.abs(b).max())
                    if phase == 0:
                        up = new
                    else:
                        uc = new
                    W = _fix(new, norm)
                R(R_AM_ITER_PRED if phase == 0 else R_AM_ITER_CORR)
                if j < 5 and sd["active"] and sd["it_active"]:
                    k2 = f(t0 + sd["dt"], W)
            R(R_AM_PRED_END if phase == 0 else R_AM_CORR_END)
        if sd["active"] and not int(sd["it_flags"]) & 4:
            for k in keys:
                for (c, a), (_, b) in zip(_chan(k, uc[k]), _chan(k, up[k])):
                    sd.fold(c, np.abs(a - b).max())
                    sd.fold(5 + c, np.abs(b).max())
        steps = sd["step"]
        R(R_AM_FINAL)
        if sd["step"] > steps:
            Y = W
            trace.append((sd["t"], sd["dt"]))
    out = (Y, trace, int(sd["rejects"]), int(sd["status"]))
    sd.close()
    return out


def _am_case():
    from oracle import fields as F
    from oracle.model import Model, Spec
    ms = 8e5
    lex = float(np.sqrt(2 * 1.3e-11 / (F.MU0 * ms * ms)))
    kw = dict(size=(1, 8, 16), cellsize=(3e-9, 3.9e-9, 3.9e-9), msat0T0=ms, lex=lex,
              gamma_ll=F.GAMMA0 / (1 + 0.02 ** 2), alpha=(0.02,) * 3, b_ext=(0.0, 0.012, 0.016), demag=True,
              normalize=True)
    m = np.random.default_rng(4).normal(size=(3,) + kw["size"])
    m /= np.sqrt((m * m).sum(0))
    return Model(Spec(**kw)), {"m": m}


def _ttm_case():
    from oracle import fields as F
    from oracle.model import Model, Spec
    ms = 8e5
    kw = dict(size=(1, 8, 16), cellsize=(4e-9,) * 3, msat0T0=ms, lex=float(np.sqrt(2 * 1.3e-11 / (F.MU0 * ms * ms))),
              gamma_ll=F.GAMMA0 / (1 + 0.02 ** 2), alpha=(0.02,) * 3, b_ext=(0.02, 0.0, 0.0), demag=True, llb=True,
              tc=630.0, spin_j=0.5, n_spins=ms / (2 * F.MUB * 0.5), temperature=300.0, ttm=True, gamma_e=700.0,
              c_l=3e6, g_ep=6e17, k_e=90.0, k_l=0.0, laser_p0=5e20, laser_t0=2e-14, laser_fwhm=1e-13,
              laser_sigma=20e-9)
    rng = np.random.default_rng(5)
    size = kw["size"]
    me = F.equilibrium_m(300.0, 630.0, 0.5)
    m = rng.normal(size=(3,) + size)
    m = me * m / np.sqrt((m * m).sum(0))
    return Model(Spec(**kw)), {"m": m, "Te": np.full(size, 300.0), "Tl": np.full(size, 300.0)}


@pytest.mark.parametrize("case", ["llg", "ttm"])
def test_am12_launch_sequence_takes_the_oracles_steps(rules, case):
    from oracle.solvers import Integrator
    model, y0 = _am_case() if case == "llg" else _ttm_case()
    keys = list(y0)
    abs_err = {k: 1e-5 if k == "m" else 1e-3 for k in keys}
    rel_err = {k: 1e-5 if k == "m" else 1e-4 for k in keys}
    dt0, nsteps = 1e-16, 25
    it = Integrator(model, y0, "am12", dt0, mindt=1e-22, maxdt=1e-12, maxabserr=abs_err, maxrelerr=rel_err)
    want = []
    for _ in range(nsteps):
        it.step()
        want.append((it.t, it.dt))
    Y, got, rejects, status = emulate_am12(rules, model, y0, dt0, nsteps, 1e-22, 1e-12, abs_err, rel_err)
    assert status == 0 and len(got) == nsteps
    for (tg, dg), (tw, dw) in zip(got, want):
        assert tg == pytest.approx(tw, rel=1e-6) and dg == pytest.approx(dw, rel=1e-5)
    assert rejects == it.bad_steps
    # the oracle keeps the raw corrector result (the reference renormalises m at its next
    # update); the device stores it renormalised
    want_y = _fix(it.y, model.s.normalize)
    for k in keys:
        assert np.abs(Y[k] - want_y[k]).max() <= 1e-9 * max(1.0, np.abs(want_y[k]).max())


def emulate_bdf(lib, model, y0, dt, nsteps, max_iter_err, max_iter):
    """enqueue_attempt's SOLVER_BDF_EULER sequence for nsteps fixed steps."""
    f, norm = model.rhs, model.s.normalize
    keys = [k for k in ("m", "Te", "Tl") if k in y0]
    sd = HostWord(lib, dt=dt)
    Y = {k: np.array(v, dtype=np.float64) for k, v in y0.items()}
    R = lambda which, eq=0: sd.rule(which, max_iter_err=max_iter_err, max_iter=max_iter, neq=len(keys), eq=eq)
    for _ in range(nsteps):
        t, h = sd["t"], sd["dt"]
        k0 = f(t, Y)
        W = dict(Y)
        for q, key in enumerate(keys):
            R(R_BDF_BEGIN, q)
            W = _fix(dict(W, **{key: Y[key] + h * k0[key]}), norm and q == 0)
            k0 = f(t + h, W)
            for j in range(max_iter + 1):
                if sd["active"] and sd["it_active"]:
                    new = Y[key] + h * k0[key]
                    for (c, a), (_, b) in zip(_chan(key, W[key]), _chan(key, new)):
                        sd.fold(c, np.abs(a - b).max())
                        sd.fold(5 + c, np.abs(a + b).max())
                    W = _fix(dict(W, **{key: new}), norm and q == 0)
                R(R_BDF_ITER, q)
                if sd["active"] and sd["rhs_due"]:
                    k0 = f(t + h, W)
                R(R_BDF_CLEAR, q)
        if not sd["active"]:
            break
        Y = W
        sd["t"] = t + h
    out = (Y, int(sd["status"]))
    sd.close()
    return out


@pytest.mark.parametrize("case", ["llg", "ttm"])
def test_bdf_euler_launch_sequence_matches_oracle(rules, case):
    from oracle.solvers import Integrator
    model, y0 = _am_case() if case == "llg" else _ttm_case()
    # in LLG mode the sweeps compare the renormalised previous iterate with the raw new one, and
    # the relaxation term's part along m makes them differ by ~dt gamma lambda |H|: the iterator
    # error stalls near 1e-5 at 0.5 fs here (1e-4 target); the two-temperature case converges
    dt, nsteps = 5e-16, 12
    tol = 1e-4 if case == "llg" else 1e-6
    it = Integrator(model, y0, "bdf_euler", dt, max_iter=8, max_iter_err=tol)
    it.run_steps(nsteps)
    Y, status = emulate_bdf(rules, model, y0, dt, nsteps, tol, 8)
    assert status == 0
    for k in y0:
        assert np.abs(Y[k] - it.y[k]).max() <= 1e-12 * max(1.0, np.abs(it.y[k]).max())


def test_bdf_euler_too_few_sweeps_stops_like_the_reference(rules):
    """More sweeps than max_iter: the oracle raises (the reference panics), the device rule
    stops the run with status 4."""
    from oracle.solvers import Integrator
    model, y0 = _am_case()
    with pytest.raises(RuntimeError, match="cannot converge"):
        Integrator(model, y0, "bdf_euler", 5e-14, max_iter=1, max_iter_err=1e-12).step()
    _, status = emulate_bdf(rules, model, y0, 5e-14, 1, 1e-12, 1)
    assert status == 4


def test_second_order_relaxation_terms_match_oracle(rules):
    """hsb_llbar02 (the fused kernel's llbar/damping/{nonconservative,conservative}/02/local)
    against the oracle's restatement of llbar-local02nc.cu and llbar-local02c.cu."""
    from oracle import fields as F
    f = rules.llbar02_host
    P3 = ctypes.c_float * 3
    f.argtypes = [ctypes.POINTER(ctypes.c_float)] * 2 + [ctypes.c_float] + [ctypes.POINTER(ctypes.c_float)] * 3
    f.restype = None
    rng = np.random.default_rng(3)
    for _ in range(200):
        m = rng.normal(size=3)
        m /= np.linalg.norm(m)
        H = rng.normal(size=3) * 1e5
        mu_par, mu_perp = rng.uniform(0, 0.01, 3), rng.uniform(0, 0.01, 3)
        g = 2.2e5
        k = P3()
        f(P3(*m), P3(*H), g, P3(*mu_par), P3(*mu_perp), k)
        want = (F.llbar_local02nc(m[:, None], H[:, None], None, None, mu_par, g) +
                F.llbar_local02c(m[:, None], H[:, None], None, None, mu_perp, g))[:, 0]
        assert np.abs(np.array(list(k)) - want).max() <= 1e-5 * np.abs(want).max()


def _f32_sweeper(lib):
    f = lib.imp_sweep_host
    fp = ctypes.POINTER(ctypes.c_float)
    dp = ctypes.POINTER(ctypes.c_double)
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_long, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                  fp, fp, fp, fp, fp, dp, dp, dp, dp, dp, fp, fp, ctypes.POINTER(ctypes.c_int)]
    f.restype = None
    P = lambda a: None if a is None else a.ctypes.data_as(dp if a.dtype == np.float64 else fp)

    def sweep(mode, ch, dt, c0, c1, normalize, y0, w, prev, dy, k0, w64=None, prev64=None, u64=None, up64=None,
              uc64=None):
        dmax = np.zeros(5, np.float32)
        smax = np.zeros(5, np.float32)
        bad = ctypes.c_int()
        f(ch, mode, y0.shape[1], dt, c0, c1, normalize, P(y0), P(w), P(prev), P(dy), P(k0), P(w64), P(prev64), P(u64),
          P(up64), P(uc64), P(dmax), P(smax), ctypes.byref(bad))
        return dmax, smax, bad.value
    return sweep


def emulate_am12_kernel(lib, model, y0, dt, nsteps, mindt, maxdt, abs_err, rel_err, t_stop=0.0):
    """enqueue_attempt's SOLVER_AM12 sequence with the sweep kernel's own cell code on the
    device's buffers (channels x cells): FP32 state, derivatives and right-hand-side iterate,
    FP64 iterates compared by the sweeps; the right-hand sides are the oracle's, rounded to FP32
    as the stage kernels store them."""
    sweep = _f32_sweeper(lib)
    keys = [k for k in ("m", "Te", "Tl") if k in y0]
    ch = 5 if len(keys) == 3 else 3
    size = y0["m"].shape[1:]
    n = int(np.prod(size))
    norm = int(model.s.normalize)
    pack = lambda d: np.ascontiguousarray(np.concatenate([np.asarray(d[k], np.float64).reshape(-1, n) for k in keys]),
                                          dtype=np.float32)

    def unpack(a):
        out = {"m": a[:3].astype(np.float64).reshape((3,) + size)}
        if ch == 5:
            out["Te"] = a[3].astype(np.float64).reshape(size)
            out["Tl"] = a[4].astype(np.float64).reshape(size)
        return out
    f = lambda t, a: pack(model.rhs(t, unpack(a)))
    neq = len(keys)
    ab = [abs_err[k] for k in keys] + [1.0] * (3 - neq)
    rl = [rel_err[k] for k in keys] + [1.0] * (3 - neq)
    sd = HostWord(lib, dt=min(dt, t_stop) if t_stop > 0 else dt, mindt=mindt, maxdt=maxdt, step_stop=nsteps,
                  t_stop=t_stop)
    R = lambda which: sd.rule(which, ab, rl, neq=neq)
    Y = pack(y0)
    W = np.zeros_like(Y)
    w64, up64, uc64 = (np.zeros(Y.shape, np.float64) for _ in range(3))
    trace = []

    def fold(dmax, smax):
        for c in range(ch):
            sd.fold(c, dmax[c])
            sd.fold(5 + c, smax[c])
    while sd["active"]:
        t0 = sd["t"]
        R(R_AM_BEGIN)
        k0 = f(t0, Y)
        sweep(AM_EULER, ch, sd["dt"], 0, ch, norm, Y, W, W, None, k0, w64)
        k1 = f(t0 + sd["dt"], W)
        k2 = np.zeros_like(k1)
        for phase in (0, 1):
            for j in range(6):
                if sd["active"] and sd["it_active"]:
                    mode = AM_PRED if phase == 0 else AM_CORR
                    dy = k2 if sd["dysel"] else k1
                    prev64 = up64 if (phase == 1 and sd["prevsel"]) else w64
                    d, s_, _ = sweep(mode, ch, sd["dt"], 0, ch, norm, Y, W, W, dy, k0, w64, prev64,
                                     up64 if phase == 0 else uc64)
                    fold(d, s_)
                R(R_AM_ITER_PRED if phase == 0 else R_AM_ITER_CORR)
                if j < 5 and sd["active"] and sd["it_active"]:
                    k2 = f(t0 + sd["dt"], W)
            R(R_AM_PRED_END if phase == 0 else R_AM_CORR_END)
        if sd["active"] and not int(sd["it_flags"]) & 4:
            d, s_, _ = sweep(AM_ERR, ch, sd["dt"], 0, ch, norm, Y, W, W, k1, k0, up64=up64, uc64=uc64)
            fold(d, s_)
        steps = sd["step"]
        R(R_AM_FINAL)
        if sd["step"] > steps:
            Y = W.copy()
            trace.append((sd["t"], sd["dt"]))
    out = (unpack(Y), trace, int(sd["status"]))
    sd.close()
    return out


@pytest.mark.parametrize("case,tol", [("llg", (1e-4, 1e-3)), ("llg", (1e-5, 1e-5)), ("ttm", (1e-4, 1e-3)),
                                      ("ttm", (1e-5, 1e-5))])
def test_am12_with_the_sweep_kernels_cell_code(rules, case, tol):
    """The same launch sequence with the sweep kernel's own per-cell code on the device's buffers
    (FP32 state and derivatives, FP64 iterates), to the same end time as the oracle: the same
    number of steps, and the state within the FP32 rounding that the steps accumulate.  Below the
    reference's default tolerances (1e-5 / 1e-5 for an LLG film, about 1400 steps) the sweeps'
    comparisons of FP64 iterates keep the oracle's step sequence, which comparisons of FP32
    iterates (rounding about 6e-8 of |m|) did not."""
    from oracle.solvers import Integrator
    model, y0 = _am_case() if case == "llg" else _ttm_case()
    keys = list(y0)
    abs_err = {k: tol[0] if k == "m" else 1e-2 for k in keys}
    rel_err = {k: tol[1] if k == "m" else 1e-3 for k in keys}
    t_end = 2e-13 if tol[0] > 5e-5 else 5e-14
    it = Integrator(model, y0, "am12", 1e-16, mindt=1e-22, maxdt=1e-12, maxabserr=abs_err, maxrelerr=rel_err)
    it.run_until(t_end)
    Y, trace, status = emulate_am12_kernel(rules, model, y0, 1e-16, -1, 1e-22, 1e-12, abs_err, rel_err, t_stop=t_end)
    assert status == 0
    assert len(trace) == it.step_count
    assert trace[-1][0] == pytest.approx(t_end, rel=1e-9)
    want = _fix(it.y, model.s.normalize)
    assert np.abs(Y["m"] - want["m"]).max() < (5e-6 if len(trace) > 1000 else 1e-6)
    if "Te" in keys:
        assert np.abs(Y["Te"] - want["Te"]).max() < 1e-6 * np.abs(want["Te"]).max()
