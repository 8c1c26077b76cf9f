"""The product's FP64 drop-in library under hotspin's own call sequence.

``oracle/replay.py`` issues, for each right-hand side and solver stage, the calls the Go
updaters issue through cgo (exchange6Async, copyPad3DAsync + FFT + tensSYMMVecMul +
copyUnPad3DAsync, vecMaddAsync, long_field_async, llbar_torque_async, Qspat_async, madd*,
partialMaxAbsAsync / partialMaxDiffAsync, normalizeAsync, ...).  Pointed at libhsb200.so
instead of the reference's libhotspin.so, the same replay must produce the same results:
that is what a Go build linking the drop-ins would compute.  Both are timed side by side.
"""
import os
import time

import numpy as np
import pytest

from oracle import fields as F
from oracle import replay
from oracle.model import Model, Spec
from tests.gpu_util import rel_err

pytestmark = pytest.mark.gpu

def _hsb():
    """The product library this process binds (libhsb200.so)."""
    from hotspin_b200 import _lib
    return _lib.load()._name
KW = dict(size=(2, 32, 64), cellsize=(4e-9, 4e-9, 4e-9), msat0T0=8e5,
          lex=float(np.sqrt(2 * 1.3e-11 / (F.MU0 * 8e5 ** 2))), gamma_ll=2.2e5, alpha=(0.02, 0.03, 0.04),
          ku=3e4, anis_u=(0.2, 0.3, 1.0), b_ext=(0.01, -0.02, 0.015), demag=True, llb=True, tc=630.0, spin_j=0.5,
          n_spins=8e5 / (2 * F.MUB * 0.5), temperature=300.0, ttm=True, gamma_e=700.0, c_l=3e6, g_ep=6e17,
          k_e=90.0, k_l=0.0, laser_p0=5e20, laser_t0=1e-13, laser_fwhm=1e-13, laser_sigma=30e-9)


def _state(size, seed=8):
    rng = np.random.default_rng(seed)
    m = rng.normal(size=(3,) + size)
    m = m / np.sqrt((m * m).sum(0)) * rng.uniform(0.5, 0.95, size=size)
    return {"m": m, "Te": rng.uniform(300, 900, size=size), "Tl": rng.uniform(300, 400, size=size)}


def test_dropins_give_the_reference_rhs_under_the_go_sequence(cuda):
    y = _state(KW["size"])
    want = Model(Spec(**KW)).rhs(0.7e-13, y)
    outs = {}
    libs = {"hsb": _hsb()}
    if replay.available():
        libs["ref"] = None
    for name, path in libs.items():
        sim = replay.RefSim(KW, dt=1e-15, lib_path=path)
        for k, v in y.items():
            sim.set(k, v)
        out = cuda.zeros_like(sim.y)
        sim.rhs(0.7e-13, sim.y, out)
        outs[name] = out.cpu().numpy().reshape((5,) + KW["size"])
    got = outs["hsb"]
    assert rel_err(got[:3], want["m"]) < 1e-11
    assert rel_err(got[3], want["Te"]) < 1e-11
    assert rel_err(got[4], want["Tl"]) < 1e-11
    if "ref" in outs:
        assert rel_err(got, outs["ref"]) < 1e-11


@pytest.mark.parametrize("solver", ["dp45", "rk12"])
def test_dropins_step_like_the_reference_library(cuda, solver):
    if not replay.available():
        pytest.skip("oracle/_ref/libhotspin.so not built (needs the reference sources)")
    kw = dict(KW, ttm=False, laser_p0=0.0, llb=False, temperature=0.0, normalize=solver == "rk12")
    rng = np.random.default_rng(9)
    m = rng.normal(size=(3,) + kw["size"])
    m /= np.sqrt((m * m).sum(0))
    res = {}
    for name, path in (("ref", None), ("hsb", _hsb())):
        sim = replay.RefSim(kw, dt=1e-15, rtol=1e-4, lib_path=path)
        sim.set("m", m)
        cuda.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(10):
            if solver == "dp45":
                sim.step()
            else:
                sim.step_rk12({"m": 1e-4})
        cuda.cuda.synchronize()
        res[name] = (sim.get("m"), sim.t, sim.attempts, time.perf_counter() - t0)
    print("\n[drop-in replay %s] reference library %.1f ms/step, libhsb200 drop-ins %.1f ms/step"
          % (solver, res["ref"][3] * 100, res["hsb"][3] * 100))
    assert res["hsb"][1] == pytest.approx(res["ref"][1], rel=1e-9)
    assert res["hsb"][2] == res["ref"][2]
    assert np.abs(res["hsb"][0] - res["ref"][0]).max() < 1e-9
