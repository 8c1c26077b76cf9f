"""The FP64 Newell tensor option on the GPU (k_newell_kernel + the plan's FP64 transforms):
its kernel spectrum and demag field against the oracle's Newell restatement, and the field's
difference from the Kernel_Arne plan (the reference's tensor), which is reported."""
import ctypes

import numpy as np
import pytest

from hotspin_b200 import _lib
from hotspin_b200.sim import Simulation, demag_plan
from oracle import demag, native
from oracle import newell as N
from tests.gpu_util import dev, host, ptr, rel_err
from tests.test_gpu_demag import _kernel_host

pytestmark = pytest.mark.gpu

GEOMS = [((1, 16, 32), (3e-9, 3.9e-9, 3.9e-9), (0, 0, 0)), ((4, 8, 16), (2e-9, 2e-9, 2e-9), (0, 0, 0)),
         ((2, 8, 16), (5e-9, 2.5e-9, 1e-9), (0, 0, 0)), ((1, 16, 16), (2e-9, 2e-9, 2e-9), (0, 2, 2))]


@pytest.mark.parametrize("size,cs,pbc", GEOMS)
def test_newell_spectrum_and_field_match_oracle(cuda, size, cs, pbc):
    logic = demag.pad_size(size, pbc)
    Kn = N.newell_kernel_full(logic, cs, pbc)
    Kf = demag.kernel_spectrum(Kn)
    rng = np.random.default_rng(4)
    m = rng.normal(size=(3,) + size)
    m /= np.sqrt((m * m).sum(0))
    want = demag.demag_field(m, None, 8e5, Kf, logic) / demag.MU0
    plan = demag_plan(size, cs, pbc, tensor="newell")
    arne = demag_plan(size, cs, pbc)
    try:
        assert rel_err(_kernel_host(plan, logic), Kf) < 2e-6
        dm = dev(cuda, m, np.float32)
        H = cuda.empty_like(dm)
        _lib.check(_lib.load().hsb_demag_field(plan, ptr(dm), None, 8e5, ptr(H), None))
        got = host(cuda, H)
        assert rel_err(got, want) < 2e-5
        Ha = cuda.empty_like(dm)
        _lib.check(_lib.load().hsb_demag_field(arne, ptr(dm), None, 8e5, ptr(Ha), None))
        d = rel_err(got, host(cuda, Ha))
        print("\n[newell vs Kernel_Arne field] %s: max |dH| / max |H| = %.1e" % (size, d))
        assert d < 5e-3
    finally:
        _lib.load().hsb_demag_plan_destroy(plan)
        _lib.load().hsb_demag_plan_destroy(arne)


def test_simulation_with_newell_tensor(cuda):
    ms = 8e5
    kw = dict(size=(2, 16, 32), cellsize=(3e-9,) * 3, msat0T0=ms,
              lex=float(np.sqrt(2 * 1.3e-11 / (4e-7 * np.pi * ms * ms))), gamma_ll=2.211e5, alpha=(0.1,) * 3,
              demag=True, normalize=True, solver="rk4", dt=1e-14)
    m = np.random.default_rng(5).normal(size=(3,) + kw["size"])
    m /= np.sqrt((m * m).sum(0))
    with Simulation(**kw, demag_tensor="newell") as a, Simulation(**kw) as b:
        a.set("m", m)
        b.set("m", m)
        Ha, Hb = a.get("H_demag"), b.get("H_demag")
        assert 0 < rel_err(Ha, Hb) < 5e-3
        a.step(10)
        assert np.isfinite(a.get("m")).all()
