"""The device step-control rules, compiled for the host, against the oracle's restatement of
hotspin's solvers (no GPU needed).

``tests/native/rule_check.cu`` includes the same inline rule the rk12 controller kernel runs
(``hsb_rk12_rule`` in ``hsb_llg.cuh``); it is built here with nvcc as host code and driven
through ctypes on random and boundary error sequences.
"""
import ctypes
import math
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle.solvers import rk12_rule

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else shutil.which("nvcc")


@pytest.fixture(scope="module")
def rules(tmp_path_factory):
    if not NVCC:
        pytest.skip("nvcc is not available")
    out = str(tmp_path_factory.mktemp("rules") / "rule_check.so")
    cmd = [NVCC, "-x", "cu", "-std=c++17", "-O2", "-Xcompiler", "-fPIC", "-shared",
           "-I" + os.path.join(ROOT, "hotspin_b200", "csrc"), os.path.join(ROOT, "tests", "native", "rule_check.cu"),
           "-o", out]
    subprocess.run(cmd, check=True, capture_output=True)
    lib = ctypes.CDLL(out)
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
