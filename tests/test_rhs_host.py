"""The generic stage kernel's per-cell right-hand side, built for the host, against the FP64 oracle.

`rhs_cell` (hotspin_b200/csrc/hsb_rhs.cuh) is the arithmetic of every generic stage launch:
exchange with its masks, anisotropy, Zeeman (constant or pointwise), the demag field input, the
MFA longitudinal field, the Philox thermal field, the LLBar torque and zero-order local
relaxation, the second-order local terms (02nc / 02c), the non-local term (two passes, the first
storing H_eff) and the two-temperature model with its laser.  tests/native/rule_check.cu runs it
over a grid with the physics the library derives from the descriptor (`phys_from_desc`,
hsb_desc.h) on FP32 buffers; the oracle (oracle/model.py) evaluates the same state in FP64.
The bound is the one the device tests use (3e-5 of the largest entry).
"""
import ctypes

import numpy as np
import pytest

from hotspin_b200.sim import make_desc
from oracle import fields as F
from oracle.model import Model, Spec

MS, AEX = 8e5, 1.3e-11
LEX = float(np.sqrt(2 * AEX / (F.MU0 * MS * MS)))
LLG = dict(size=(2, 16, 32), cellsize=(3e-9, 3.9e-9, 3.9e-9), msat0T0=MS, lex=LEX,
           gamma_ll=F.GAMMA0 / (1 + 0.02 ** 2), alpha=(0.02, 0.02, 0.02), b_ext=(0.0, 0.012, 0.016),
           demag=True, normalize=True, ku=2e4, anis_u=(0.3, 0.0, 1.0))
LLB = dict(size=(4, 16, 16), cellsize=(2e-9, 2e-9, 2e-9), msat0T0=1.1e6,
           lex=float(np.sqrt(2 * 1e-11 / (F.MU0 * 1.1e6 ** 2))), gamma_ll=F.GAMMA0, alpha=(0.1, 0.1, 0.1), ku=7e6,
           anis_u=(1.0, 0.0, 0.0), demag=True, llb=True, tc=700.0, spin_j=0.5, n_spins=1.1e6 / (2 * F.MUB * 0.5),
           temperature=300.0)
TTM = dict(LLB, size=(2, 16, 32), cellsize=(4e-9, 4e-9, 4e-9), msat0T0=MS, lex=LEX, tc=630.0,
           n_spins=MS / (2 * F.MUB * 0.5), alpha=(0.02, 0.02, 0.02), ku=0.0, ttm=True, gamma_e=700.0, c_l=3e6,
           g_ep=6e17, k_e=90.0, k_l=20.0, laser_p0=5e20, laser_t0=0.0, laser_fwhm=1e-13, laser_sigma=40e-9)


@pytest.fixture(scope="module")
def rhs_host(host_rules):
    f = host_rules.rhs_host
    fp = ctypes.POINTER(ctypes.c_float)
    f.argtypes = [ctypes.c_void_p, fp, fp, fp, ctypes.c_double, ctypes.c_double, ctypes.c_longlong, fp, fp, fp, fp]
    f.restype = None
    return f


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def host_rhs(f, kw, y, t=0.0, dt=1e-14, step=0, hd=None, msat_mask=None, lex_mask=None):
    """k = f(t, y) by the kernel's per-cell code; y as the oracle's state dict (program order)."""
    d = make_desc(**{k: v for k, v in kw.items() if k not in ("msat_mask", "lex_mask")})
    keys = ["m", "Te", "Tl"] if kw.get("ttm") else ["m"]
    size = tuple(kw["size"])
    n = int(np.prod(size))
    ys = _f32(np.concatenate([np.asarray(y[k], np.float64).reshape(-1, n) for k in keys]))
    k = np.zeros_like(ys)
    hbuf = np.zeros((3, n), np.float32)
    hd32 = _f32(None if hd is None else hd.reshape(3, n))
    ms32, lx32 = _f32(msat_mask), _f32(lex_mask)
    f(ctypes.byref(d), _p(ys), _p(hd32), _p(ys), t, dt, step, _p(ms32), _p(lx32), _p(hbuf), _p(k))
    out = {"m": k[:3].astype(np.float64).reshape((3,) + size)}
    if kw.get("ttm"):
        out["Te"] = k[3].astype(np.float64).reshape(size)
        out["Tl"] = k[4].astype(np.float64).reshape(size)
    return out


def state(kw, seed=5):
    size = tuple(kw["size"])
    rng = np.random.default_rng(seed)
    m = rng.normal(size=(3,) + size)
    m /= np.sqrt((m * m).sum(0))
    y = {}
    if kw.get("llb"):
        m = m * rng.uniform(0.6, 0.95, size=size)
    y["m"] = m
    if kw.get("ttm"):
        y["Te"] = rng.uniform(300.0, 900.0, size=size)
        y["Tl"] = rng.uniform(300.0, 400.0, size=size)
    return y


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def compare(f, kw, y, t=0.0, dt=1e-14, step=0, tol=3e-5):
    spec = Spec(**kw)
    model = Model(spec)
    model.set_thermal(step, dt, model.spin_temperature(y))
    want = model.rhs(t, y)
    hd = None
    if spec.demag:
        m = F.normalize(y["m"]) if spec.normalize else y["m"]
        hd = model.plan.field(m, spec.msat_mask, spec.msat0T0) / F.MU0
    yy = dict(y, m=F.normalize(y["m"])) if spec.normalize else y
    got = host_rhs(f, kw, yy, t, dt, step, hd, spec.msat_mask, spec.lex_mask)
    for key in want:
        assert rel(got[key], want[key]) < tol, (key, rel(got[key], want[key]))
    return got, want


@pytest.mark.parametrize("kw", [LLG, LLB, TTM], ids=["llg", "llb", "ttm"])
@pytest.mark.parametrize("thermal", [False, True])
def test_rhs_cell_matches_oracle(rhs_host, kw, thermal):
    kw = dict(kw, thermal=thermal, seed=77)
    if thermal and not kw.get("llb"):
        kw["temperature"] = 200.0
    compare(rhs_host, kw, state(kw), t=3e-14, step=5)


def test_rhs_cell_thermal_stream_is_the_oracles(rhs_host):
    """Thermal field alone (no other term): the kernel's Philox normals and amplitude are the
    oracle's stream, step after step (FP32 Box-Muller against FP64)."""
    kw = dict(size=(1, 8, 16), cellsize=(3e-9,) * 3, msat0T0=MS, gamma_ll=F.GAMMA0, alpha=(0.1, 0.2, 0.3),
              normalize=True, thermal=True, seed=123456789012, temperature=300.0)
    y = state(kw, seed=8)
    for step in (0, 1, 2, 1 << 33):
        compare(rhs_host, kw, y, dt=2e-14, step=step, tol=2e-5)


def test_rhs_cell_with_masks(rhs_host):
    size = (2, 8, 16)
    rng = np.random.default_rng(4)
    ms = rng.uniform(0.3, 1.0, size=size)
    ms[0, 3:5, 3:6] = 0.0
    lex = 1.0 / np.maximum(ms, 0.3)
    kw = dict(LLG, size=size, msat_mask=ms, lex_mask=lex)
    got, _ = compare(rhs_host, kw, state(kw))
    assert np.all(got["m"][:, 0, 3:5, 3:6] == 0.0)


@pytest.mark.parametrize("kw", [LLG, LLB], ids=["llg", "llb"])
def test_rhs_cell_second_order_terms(rhs_host, kw):
    kw = dict(kw, mu_par=(0.02, 0.015, 0.01), mu_perp=(0.005, 0.01, 0.02))
    compare(rhs_host, kw, state(kw, seed=23))


@pytest.mark.parametrize("pbc", [(0, 0, 0), (0, 2, 3), (1, 1, 1)])
def test_rhs_cell_nonlocal_term(rhs_host, pbc):
    """Two passes as on the device: H_eff of every cell stored, then its Laplacian with clamped
    or wrapped neighbours."""
    kw = dict(LLG, pbc=pbc, alpha_e=(2e-19, 3e-19, 1e-19))
    if pbc == (1, 1, 1):
        kw["demag"] = False
    compare(rhs_host, kw, state(kw, seed=29))


def test_rhs_cell_pointwise_tables(rhs_host):
    """Pointwise laser profile and applied field (piecewise linear in time) at several times,
    inside and outside the tables' ranges."""
    tab = [(0.0, 0.0), (5e-14, 1.0), (1.5e-13, 0.3), (3e-13, 0.0)]
    btab = [(0.0, 0.0, 0.0, 0.0), (1e-13, 0.05, -0.02, 0.01), (4e-13, -0.03, 0.04, 0.0)]
    kw = dict(TTM, laser_table=tab, bext_table=btab)
    y = state(kw, seed=3)
    for t in (-1e-14, 0.0, 3e-14, 1e-13, 2.7e-13, 5e-13):
        compare(rhs_host, kw, y, t=t)


def test_rhs_cell_langevin_and_high_spin(rhs_host):
    """The longitudinal field with a classical (Langevin) spin and with J = 7/2."""
    for J in (3.5, 1e6):
        kw = dict(LLB, spin_j=J, n_spins=1.1e6 / (2 * F.MUB * min(J, 1e3)))
        compare(rhs_host, kw, state(kw, seed=int(J) % 97))
