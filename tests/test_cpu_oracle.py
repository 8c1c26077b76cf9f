"""CPU checks of the oracle's building blocks."""
import numpy as np
import pytest

from oracle import dump, fields, philox
from oracle.model import Model, Spec
from oracle.solvers import Integrator


def test_philox_known_answers():
    # published known-answer vectors of Philox4x32-10
    cases = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
             ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
             ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
              (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]
    for ctr, key, want in cases:
        r = philox.philox4x32_10([np.array([c], dtype=np.uint32) for c in ctr], key)
        assert tuple(int(x[0]) for x in r) == want


def test_thermal_normals_statistics():
    g = philox.thermal_normals(200000, 7, 12345)
    assert abs(g.mean()) < 0.01 and abs(g.std() - 1) < 0.01
    assert abs(np.corrcoef(g[0], g[1])[0, 1]) < 0.01


def test_dump_roundtrip(tmp_path):
    a = np.random.default_rng(0).normal(size=(3, 2, 3, 4)).astype(np.float32)
    p = tmp_path / "x.dump"
    dump.write_dump(str(p), a, cellsize=(1e-9, 2e-9, 3e-9), label="m")
    b, h = dump.read_dump(str(p))
    assert np.array_equal(a.astype(np.float64), b) and h["crc"] != 0
    raw = bytearray(p.read_bytes())
    raw[200] ^= 1
    p.write_bytes(bytes(raw))
    with pytest.raises(ValueError):
        dump.read_dump(str(p))


def test_brillouin_half_spin_is_tanh():
    x = np.linspace(-3, 3, 101)
    assert np.allclose(fields.brillouin(0.5, x), np.tanh(x), atol=1e-12)
    assert np.allclose(fields.dbrillouin(0.5, x), 1 - np.tanh(x) ** 2, atol=1e-9)


def test_equilibrium_m_root():
    me = fields.equilibrium_m(300.0, 700.0, 0.5)
    b = 3 * (0.5 / 1.5) * 700.0 / 300.0
    assert abs(np.tanh(b * me) - me) < 1e-7 and 0.5 < me < 1.0
    assert fields.equilibrium_m(800.0, 700.0, 0.5) == 0.0


def test_pointwise_of_linear_interpolation():
    pts = [(0.0, 1.0), (1.0, 3.0), (3.0, -1.0)]
    assert fields.pointwise_of(pts, 0.5) == [2.0]
    assert fields.pointwise_of(pts, 2.0) == [1.0]
    assert fields.pointwise_of(pts, 3.0) == [-1.0]
    with pytest.raises(ValueError):
        fields.pointwise_of(pts, 4.0)


def test_rk4_fourth_order_on_precession():
    """Single cell in a field, no damping: RK4 error falls ~16x per halving of dt."""
    spec = Spec(size=(1, 1, 1), cellsize=(1e-9,) * 3, b_ext=(0.0, 0.0, 0.1), alpha=(0, 0, 0))
    errs = []
    for dt in (2e-12, 1e-12):
        m0 = {"m": np.array([1.0, 0.0, 0.0]).reshape(3, 1, 1, 1)}
        it = Integrator(Model(spec), m0, "rk4", dt)
        n = int(round(4e-11 / dt))
        it.run_steps(n)
        w = spec.gamma_ll * 0.1 / fields.MU0
        # hotspin's torque is +gamma (m x H): m precesses clockwise about +z
        want = np.array([np.cos(w * 4e-11), -np.sin(w * 4e-11)])
        errs.append(np.abs(it.y["m"][:2, 0, 0, 0] - want).max())
    assert 12 < errs[0] / errs[1] < 20


def test_dp45_reaches_tolerance():
    spec = Spec(size=(1, 1, 1), cellsize=(1e-9,) * 3, b_ext=(0.0, 0.0, 0.1), alpha=(0.1, 0.1, 0.1))
    it = Integrator(Model(spec), {"m": np.array([1.0, 0.0, 0.0]).reshape(3, 1, 1, 1)}, "dp45", 1e-13,
                    rtol=1e-8)
    while it.t < 1e-10:
        it.step()
    assert it.step_count > 5 and it.dt > 1e-13
