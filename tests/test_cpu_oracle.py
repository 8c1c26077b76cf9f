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


def test_debye_cp_restatement():
    """Trapezoid Debye integral: close to the exact integral, the T << Td limit, zero Td."""
    from scipy.integrate import quad
    T = np.array([[[5.0, 150.0, 300.0, 2000.0]]])
    Td = np.full(T.shape, 300.0)
    got = fields.debye_cp(T, Td, None, 1.0)
    for v, t in zip(got.ravel(), T.ravel()):
        u = 300.0 / t
        exact = quad(lambda x: x ** 4 * np.exp(x) / np.expm1(x) ** 2 if x > 0 else 0.0, 0, u)[0] / u ** 3
        assert abs(v - exact) < 2e-3 * exact
    # high-temperature limit: (T/Td)^3 * (Td/T)^3 / 3 -> 1/3
    assert abs(got.ravel()[-1] - 1.0 / 3.0) < 2e-3
    low = fields.debye_cp(np.array([[[1.0]]]), np.array([[[300.0]]]), None, 1.0).ravel()[0]
    assert abs(low - 4 * np.pi ** 4 / 15 / 300.0 ** 3) < 1e-12 * low
    assert fields.debye_cp(np.array([[[10.0]]]), np.array([[[0.0]]]), None, 1.0).ravel()[0] == 0.0


def test_spin_temperature_inverts_equilibrium():
    """Ts(m_e(T)) = T for the mean-field equilibrium (J = 1/2 and 7/2)."""
    for S in (0.5, 3.5):
        for T in (100.0, 350.0, 600.0):
            me = fields.equilibrium_m(T, 630.0, S)
            ts = fields.spin_temperature(np.array([[[me]]]), None, None, None, 1.0, 1.0, 630.0, S, (1, 1, 1))
            assert abs(ts.ravel()[0] - T) < 1e-5 * T
    edge = fields.spin_temperature(np.array([[[0.0, 1.0]]]), None, None, None, 1.0, 1.0, 630.0, 0.5, (1, 1, 2))
    assert edge.ravel().tolist() == [630.0, 0.0]


def test_weighted_avg_energy_flow_nonlocal():
    a, b = np.array([400.0, 300.0, 1.0]), np.array([400.0, 500.0, 2.0])
    w = fields.weighted_avg(a, b, None, None, None, 1.0, 1.0, 0.0)
    assert np.allclose(w, (a + b) / 2)
    w = fields.weighted_avg(a, b, np.array([1.0, 1.0, 0.0]), np.array([1.0, 1.0, 0.0]), None, 1.0, 1.0, 1.0)
    assert np.allclose(w[:2], ((np.sqrt(a) + np.sqrt(b)) / 2)[:2] ** 2) and w[2] == 0.0
    m = np.zeros((3, 1, 1, 2))
    m[2] = 1.0
    R = np.ones((3, 1, 1, 2))
    ef = fields.energy_flow(m, R, np.array([[[630.0, 0.0]]]), None, None, 0.5)
    assert np.allclose(ef.ravel(), [630.0 * 0.25 / 0.75, 0.0])
    # uniform lambda: the nonlocal term is -lambda times the Laplacian of H
    rng = np.random.default_rng(1)
    h = rng.normal(size=(3, 4, 5, 6))
    cs = (1.0, 2.0, 3.0)
    t = fields.llbar_nonlocal00nc(h, None, None, (1.0, 1.0, 1.0), cs, (1, 1, 1))
    lap = sum((np.roll(h, 1, axis=d + 1) + np.roll(h, -1, axis=d + 1) - 2 * h) / cs[d] ** 2 for d in range(3))
    assert np.allclose(t, -lap)
