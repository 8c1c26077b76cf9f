"""hotspin's script API mirrored on the B200 handle (hotspin_b200.api).

test_demag_cmp_ref follows the reference's tests/test-demag/cmp-ref.py step by step:
64^3 grid, random Msat mask and unit m from random.seed(0), load('demag'), compare B with
the reference's golden dump using its own pass criterion (absolute error per cell < 1e-6).
"""
import math
import os

import numpy as np
import pytest

from hotspin_b200 import api
from oracle import fields as F
from oracle.model import Model, Spec
from oracle.solvers import Integrator
from tests.golden.make_golden import N, demag_inputs

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _user_scalar(p):
    return np.transpose(p, (2, 1, 0))


def _user_vector(p):
    return np.stack([_user_scalar(p[2]), _user_scalar(p[1]), _user_scalar(p[0])])


def test_demag_cmp_ref(cuda):
    gold = np.load(os.path.join(HERE, "golden", "golden_subsample.npz"))
    msk_p, m_p = demag_inputs()                 # regenerated exactly as cmp-ref.py does
    msk, m = _user_scalar(msk_p), _user_vector(m_p)
    for tag, per in (("", None), ("_pbc", (8, 4, 2))):
        e = api.new_engine()
        e.setgridsize(N, N, N)
        e.setcellsize(320e-9 / N, 160e-9 / N, 64e-9 / N)
        if per:
            e.setperiodic(*per)
        e.load("llbar")
        e.load("demag")
        e.setmask("Msat0T0", msk[None])
        e.setv("Msat0T0", 800e3)
        e.setarray("m", m)
        new = e.getarray("B")
        ref = gold["B_ref%s" % tag]
        new_p = np.stack([np.transpose(new[2], (2, 1, 0)), np.transpose(new[1], (2, 1, 0)),
                          np.transpose(new[0], (2, 1, 0))]).reshape(3, -1)[:, gold["sample_flat_index"]]
        verror = np.abs(new_p - ref).sum(0).mean()       # "Absolute error per cell"
        assert verror < 1e-6, (tag, verror)
        e._reset()


def test_stdproblem4_geometry_short_run(cuda):
    """tests/stdproblem4-llbr-modular.py's module set and parameters (alpha = 0.02 stage),
    uniform start, 200 RK4 steps, against the FP64 oracle."""
    Nx, Ny, Nz = 128, 32, 1
    Ms0, Aex, alpha = 800e3, 1.3e-11, 0.02
    lex = math.sqrt(2 * Aex / (F.MU0 * Ms0 * Ms0))
    gll = 2.211e5 / (1 + alpha ** 2)
    e = api.new_engine()
    e.setgridsize(Nx, Ny, Nz)
    e.setcellsize(500e-9 / Nx, 125e-9 / Ny, 3e-9 / Nz)
    for mod in ("exchange6", "demag", "zeeman", "llbar", "llbar/torque", "llbar/damping/nonconservative/00/local",
                "normalizer", "solver/rk4"):
        e.load(mod)
    e.setv("Msat0T0", Ms0)
    e.setv("lex", lex)
    e.setv("α", [alpha] * 3)
    e.setv("γ_LL", gll)
    e.setv("B_ext", [-24.6e-3, 4.3e-3, 0.0])
    e.setv("dt", 50e-15)
    m = np.zeros((3, Nx, Ny, Nz))
    m[0] = m[1] = 1 / math.sqrt(2)
    e.setarray("m", m)
    e.step(200)
    got = e.getarray("m")
    spec = Spec(size=(Nz, Ny, Nx), cellsize=(3e-9 / Nz, 125e-9 / Ny, 500e-9 / Nx), msat0T0=Ms0, lex=lex,
                gamma_ll=gll, alpha=(alpha,) * 3, b_ext=(0.0, 4.3e-3, -24.6e-3), demag=True, normalize=True)
    mp = np.stack([np.transpose(m[2], (2, 1, 0)), np.transpose(m[1], (2, 1, 0)), np.transpose(m[0], (2, 1, 0))])
    it = Integrator(Model(spec), {"m": mp}, "rk4", 50e-15)
    it.run_steps(200)
    want = _user_vector(it.y["m"])
    assert np.abs(got - want).max() < 1e-5
    assert e.getv("t") == pytest.approx(200 * 50e-15)
    e._reset()


def test_device_array_transfers(cuda):
    """hsb_sim_set_device / hsb_sim_get_device move the state to and from caller-owned FP64
    device arrays (the layout of hotspin's gpu.Array) and equal the host transfers."""
    import ctypes

    from hotspin_b200 import _lib
    from hotspin_b200.sim import Simulation
    size = (2, 8, 16)
    rng = np.random.default_rng(21)
    m = rng.normal(size=(3,) + size)
    m /= np.sqrt((m * m).sum(0))
    with Simulation(size=size, cellsize=(2e-9,) * 3, msat0T0=8e5, solver="rk4", dt=1e-15, ttm=True, llb=True,
                    tc=630.0, spin_j=0.5, n_spins=1e28, gamma_e=700.0, c_l=3e6, temperature=300.0) as sim:
        dm = cuda.from_numpy(m).cuda()
        _lib.check(sim._lib.hsb_sim_set_device(sim._h, b"m", ctypes.c_void_p(dm.data_ptr()), dm.numel()))
        np.testing.assert_array_equal(sim.get("m"), m.astype(np.float32).astype(np.float64))
        Te = cuda.full(size, 412.5, dtype=cuda.float64, device="cuda")
        _lib.check(sim._lib.hsb_sim_set_device(sim._h, b"Te", ctypes.c_void_p(Te.data_ptr()), Te.numel()))
        back = cuda.empty((3,) + size, dtype=cuda.float64, device="cuda")
        _lib.check(sim._lib.hsb_sim_get_device(sim._h, b"m", ctypes.c_void_p(back.data_ptr()), back.numel()))
        np.testing.assert_array_equal(back.cpu().numpy(), sim.get("m"))
        assert float(sim.get("Te").max()) == 412.5
        rc = sim._lib.hsb_sim_get_device(sim._h, b"m", ctypes.c_void_p(back.data_ptr()), 7)
        assert rc == 1
