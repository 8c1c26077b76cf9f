"""Size-independent properties at the benchmark's full size (512 x 512 x 4, demag padded to
1024 x 1024 x 8) and at the large-instance size (1024 x 1024 x 32, padded 2048 x 2048 x 64),
where the FP64 oracle is too slow to run: linearity and reciprocity of the demag convolution,
the thin-film demag limit, energy conservation without damping and energy decay with damping."""
import ctypes

import numpy as np
import pytest

from hotspin_b200 import _lib
from hotspin_b200.sim import Simulation, demag_plan
from tests.gpu_util import dev, host, ptr

pytestmark = pytest.mark.gpu

SIZE = (4, 512, 512)
CS = (4e-9, 4e-9, 4e-9)
MS = 8e5
LEX = float(np.sqrt(2 * 1.3e-11 / (4e-7 * np.pi * MS * MS)))


@pytest.fixture(scope="module")
def plan(cuda):
    p = demag_plan(SIZE, CS, (0, 0, 0))
    yield p
    _lib.load().hsb_demag_plan_destroy(p)


def _field(cuda, plan, m):
    dm = dev(cuda, m, np.float32)
    H = cuda.empty_like(dm)
    _lib.check(_lib.load().hsb_demag_field(plan, ptr(dm), None, MS, ptr(H), None), "hsb_demag_field")
    return host(cuda, H).astype(np.float64)


def _unit(seed):
    m = np.random.default_rng(seed).normal(size=(3,) + SIZE)
    return m / np.sqrt((m * m).sum(0))


def test_demag_linearity_and_reciprocity(cuda, plan):
    m1, m2 = _unit(1), _unit(2)
    h1, h2 = _field(cuda, plan, m1), _field(cuda, plan, m2)
    h12 = _field(cuda, plan, 0.3 * m1 - 0.7 * m2)
    lin = np.abs(h12 - (0.3 * h1 - 0.7 * h2)).max() / np.abs(h12).max()
    assert lin < 1e-5
    # symmetric tensor: sum m1 . H(m2) = sum m2 . H(m1)
    a, b = float((m1 * h2).sum()), float((m2 * h1).sum())
    assert abs(a - b) < 1e-5 * max(abs(a), abs(b))


def test_thin_film_demag_limit(cuda, plan):
    """A uniformly magnetized 2 um x 2 um x 16 nm film: inside, H = -Ms along the normal
    (N_zz -> 1) and almost no field in the plane (N_xx -> 0)."""
    m = np.zeros((3,) + SIZE)
    m[0] = 1.0                          # program component 0 = user z = film normal
    h = _field(cuda, plan, m)
    c = (slice(None), slice(192, 320), slice(192, 320))
    assert abs(h[0][c].mean() / MS + 1.0) < 0.02
    m = np.zeros((3,) + SIZE)
    m[2] = 1.0                          # in-plane (user x)
    h = _field(cuda, plan, m)
    assert abs(h[2][c].mean() / MS) < 0.02


def test_energy_conserved_without_damping_and_decays_with_it(cuda):
    """LLG (|m| = 1) from a smooth non-uniform state: without damping RK4 keeps the energy
    constant; with damping it decreases monotonically."""
    a1 = np.arange(SIZE[1])[:, None] / SIZE[1]
    a2 = np.arange(SIZE[2])[None, :] / SIZE[2]
    th = 0.6 + 0.3 * np.sin(2 * np.pi * a1) * np.cos(2 * np.pi * a2)
    ph = 2 * np.pi * (a1 + 0.5 * a2)
    m = np.stack([np.cos(th), np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph)])
    m = np.broadcast_to(m[:, None], (3,) + SIZE).copy()
    drift = 0.0
    for alpha in (0.0, 0.5):
        with Simulation(size=SIZE, cellsize=CS, msat0T0=MS, lex=LEX, alpha=(alpha,) * 3, demag=True,
                        normalize=True, b_ext=(0.0, 0.0, 0.01), solver="rk4", dt=10e-15) as sim:
            sim.set("m", m)
            E = [sim.energy()]
            for _ in range(5):
                sim.step(40)
                E.append(sim.energy())
        E = np.array(E)
        if alpha == 0.0:
            drift = np.abs(E - E[0]).max()
            assert drift < 1e-4 * abs(E[0])
        else:
            assert np.all(np.diff(E) < 0)
            assert E[0] - E[-1] > 10 * drift


def test_multipass_demag_properties_at_large_size(cuda):
    """The multi-pass y/z path at the large-instance size (1024x1024x32 cells of 2 nm, padded
    2048x2048x64: 2048-point y columns, 64-point z convolution): linearity and reciprocity of
    the convolution, and a uniform film's interior field along its normal near -Ms."""
    size, cs = (32, 1024, 1024), (2e-9, 2e-9, 2e-9)
    lib = _lib.load()
    p = demag_plan(size, cs, (0, 0, 0))
    try:
        def field(m):
            dm = dev(cuda, m, np.float32)
            H = cuda.empty_like(dm)
            _lib.check(lib.hsb_demag_field(p, ptr(dm), None, MS, ptr(H), None), "hsb_demag_field")
            return host(cuda, H).astype(np.float64)

        rng = np.random.default_rng(9)
        m1 = rng.normal(size=(3,) + size).astype(np.float32)
        m2 = rng.normal(size=(3,) + size).astype(np.float32)
        h1, h2 = field(m1), field(m2)
        h12 = field(0.3 * m1 - 0.7 * m2)
        assert np.abs(h12 - (0.3 * h1 - 0.7 * h2)).max() / np.abs(h12).max() < 1e-5
        a, b = float((m1 * h2).sum()), float((m2 * h1).sum())
        assert abs(a - b) < 1e-5 * max(abs(a), abs(b))
        m = np.zeros((3,) + size, np.float32)
        m[0] = 1.0                     # along the thickness (program axis 0)
        h = field(m)
        core = h[0][12:20, 384:640, 384:640]
        assert -1.0 < core.mean() / MS < -0.9
    finally:
        lib.hsb_demag_plan_destroy(p)
