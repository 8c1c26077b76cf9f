"""FP64 drop-in kernels (hotspin's libhotspin.h names and signatures) against the oracle."""
import ctypes
import math
import os

import numpy as np
import pytest

from hotspin_b200 import _lib
from oracle import demag, fields, native
from tests.gpu_util import dev, host, ptr, rel_err

pytestmark = pytest.mark.gpu

D = ctypes.c_double
I = ctypes.c_int
SIZE = (6, 10, 14)
N = int(np.prod(SIZE))
CS = (2e-9, 3e-9, 5e-9)


@pytest.fixture(scope="module")
def lib(cuda):
    return _lib.load()


def rnd(shape, seed, lo=-1.0, hi=1.0):
    return np.random.default_rng(seed).uniform(lo, hi, size=shape)


def unit(seed, size=SIZE):
    m = np.random.default_rng(seed).normal(size=(3,) + size)
    return m / np.sqrt((m * m).sum(0))


def comps(t):
    return [ptr(t[c]) for c in range(t.shape[0])]


@pytest.mark.parametrize("pbc", [(0, 0, 0), (1, 0, 1), (1, 1, 1)])
@pytest.mark.parametrize("with_mask", [False, True])
def test_exchange6(lib, cuda, pbc, with_mask):
    m = unit(1)
    lex = rnd(SIZE, 2, 0.5, 2.0) if with_mask else None
    lexmul = 5.7e-9
    want = fields.exchange6(m, lex, 8e5, lexmul, CS, pbc)
    dm = dev(cuda, m)
    dh = cuda.empty_like(dm)
    dl = dev(cuda, lex) if with_mask else None
    c = [lexmul ** 2 / (x * x) for x in CS]
    lib.exchange6Async(*comps(dh), *comps(dm), None, ptr(dl), I(SIZE[0]), I(SIZE[1]), I(SIZE[2]),
                       I(pbc[0]), I(pbc[1]), I(pbc[2]), D(8e5), D(c[0]), D(c[1]), D(c[2]), None)
    assert rel_err(host(cuda, dh), want) < 1e-12


def test_uniaxial_and_torques(lib, cuda):
    m = unit(3)
    h = rnd((3,) + SIZE, 4) * 1e5
    ms = rnd(SIZE, 5, 0.0, 1.0)
    ms[0, 0, :3] = 0.0
    ku = rnd(SIZE, 6, 0.5, 1.5)
    dm, dh, dms, dku = dev(cuda, m), dev(cuda, h), dev(cuda, ms), dev(cuda, ku)
    out = cuda.empty_like(dm)
    pre = 2 * 5e5 / (fields.MU0 * 8e5)
    lib.uniaxialAnisotropyAsync(*comps(out), *comps(dm), ptr(dku), ptr(dms), D(pre), None, D(0.2), None, D(0.3),
                                None, D(0.9), None, I(N))
    want = fields.uniaxial_anisotropy(m, ku, ms, 5e5, 8e5, None, (0.2, 0.3, 0.9))
    assert rel_err(host(cuda, out), want) < 1e-12
    lib.llbar_torque_async(*comps(out), *comps(dm), *comps(dh), ptr(dms), None, I(N))
    assert rel_err(host(cuda, out), fields.llbar_torque(m, h, ms, 1.0)) < 1e-12
    lib.llbar_local00nc_async(*comps(out), *comps(dh), ptr(dms), None, None, None, D(0.1), D(0.2), D(0.3), None, I(N))
    assert rel_err(host(cuda, out), fields.llbar_local00nc(h, ms, None, (0.1, 0.2, 0.3), 1.0)) < 1e-12
    lib.llbar_local02nc_async(*comps(out), *comps(dm), *comps(dh), ptr(dms), None, None, None, D(0.1), D(0.2), D(0.3),
                              None, I(N))
    assert rel_err(host(cuda, out), fields.llbar_local02nc(m, h, ms, None, (0.1, 0.2, 0.3), 1.0)) < 1e-12
    lib.llbar_local02c_async(*comps(out), *comps(dm), *comps(dh), ptr(dms), None, None, None, D(0.1), D(0.2), D(0.3),
                             None, I(N))
    assert rel_err(host(cuda, out), fields.llbar_local02c(m, h, ms, None, (0.1, 0.2, 0.3), 1.0)) < 1e-12
    lib.normalizeAsync(*comps(dh), None, I(N))
    assert rel_err(host(cuda, dh), fields.normalize(h)) < 1e-14


@pytest.mark.parametrize("S", [0.5, 1.5, 3.5, 1e6])
def test_mfa_long_field_brillouin_kappa(lib, cuda, S):
    rng = np.random.default_rng(7)
    m = unit(8) * rng.uniform(0.05, 1.0, size=SIZE)
    # above ~50 K the reference's closed form of B_J' cancels to 0 in FP64 (both sides then
    # return inf); the parity range starts well above that
    T = rng.uniform(150.0, 640.0, size=SIZE)
    T[0, 0, 0] = 0.0
    T[0, 0, 1] = 700.0
    Tc, n = 633.0, 5.5e28
    dm, dT = dev(cuda, m), dev(cuda, T)
    out = cuda.empty_like(dm)
    lib.long_field_async(*comps(out), *comps(dm), None, None, None, None, ptr(dT), D(8e5), D(S), D(n), D(Tc), D(1.0),
                         I(N), None)
    want = fields.long_field(m, None, None, None, None, T, 8e5, S, n, Tc, 1.0)
    got = host(cuda, out)
    ok = T > 0
    assert rel_err(got[:, ok], want[:, ok]) < 1e-9
    ms0 = cuda.empty_like(dT)
    lib.brillouinAsync(ptr(ms0), None, ptr(dT), None, None, D(8e5), D(8e5), D(Tc), D(S), I(N), None)
    want_ms = fields.brillouin_msat0(T, None, None, None, 8e5, 8e5, Tc, S)
    assert rel_err(host(cuda, ms0), want_ms) < 1e-9
    kap = cuda.empty_like(dT)
    lib.kappaAsync(ptr(kap), ptr(ms0), None, ptr(dT), None, None, None, D(8e5), D(8e5), D(Tc), D(S), I(N), None)
    want_k = fields.kappa(want_ms, None, T, None, None, None, 8e5, 8e5, Tc, S)
    assert rel_err(host(cuda, kap), want_k) < 1e-6


def test_thermal_scaling(lib, cuda):
    g = np.random.default_rng(9).normal(size=(3,) + SIZE)
    T = rnd(SIZE, 10, 0.0, 600.0)
    ms = rnd(SIZE, 11, 0.0, 1.0)
    ms[1, 1, :2] = 0
    dg, dT, dms = dev(cuda, g), dev(cuda, T), dev(cuda, ms)
    pre = fields.thermal_prefactor(1.0, CS, 2.2e5, 1e-14, 0.0, 8e5)
    lib.temperature_scaleAnizNoise(*comps(dg), None, None, None, ptr(dT), ptr(dms), D(0.01), D(0.02), D(0.03), D(pre),
                                   None, I(N))
    want = fields.scale_noise(g, None, (0.01, 0.02, 0.03), T, ms, pre)
    assert rel_err(host(cuda, dg), want) < 1e-12


def test_tensor_multiply_and_pad(lib, cuda):
    size, cs = (4, 6, 8), (1e-9, 2e-9, 3e-9)
    logic = demag.pad_size(size, (0, 0, 0))
    Kf = demag.kernel_spectrum(native.kernel_arne(logic, cs, (0, 0, 0)))
    m = unit(12, size)
    # pad + forward FFT on the host, multiply on the device, compare with the oracle
    F = [np.fft.rfftn(np.pad(m[c], [(0, logic[a] - size[a]) for a in range(3)])) for c in range(3)]
    src = [dev(cuda, np.stack([f.real, f.imag], -1)) for f in F]
    dst = [cuda.empty_like(s) for s in src]
    kern = [dev(cuda, np.ascontiguousarray(Kf[c])) for c in range(6)]
    C2 = logic[2] // 2 + 1
    lib.tensSYMMVecMul(*[ptr(d) for d in dst], *[ptr(s) for s in src], *[ptr(k) for k in kern], D(2.5), I(logic[0]),
                       I(logic[1]), I(C2), None)
    K = demag.unfold_spectrum(Kf, logic)
    XX, YY, ZZ, YZ, XZ, XY = range(6)
    want = [K[XX] * F[0] + K[XY] * F[1] + K[XZ] * F[2], K[XY] * F[0] + K[YY] * F[1] + K[YZ] * F[2],
            K[XZ] * F[0] + K[YZ] * F[1] + K[ZZ] * F[2]]
    for c in range(3):
        got = host(cuda, dst[c])
        assert rel_err(got[..., 0] + 1j * got[..., 1], 2.5 * want[c]) < 1e-13
    # copyPad3D / copyUnPad3D per component (copypad.cu)
    a = rnd((3,) + size, 13)
    da = dev(cuda, a)
    big = cuda.zeros((3,) + tuple(logic), dtype=cuda.float64, device="cuda")
    lib.copyPad3DAsync(ptr(big), I(logic[0]), I(logic[1]), I(logic[2]), ptr(da), I(size[0]), I(size[1]), I(size[2]),
                       I(3), None)
    b = host(cuda, big)
    assert np.array_equal(b[:, :size[0], :size[1], :size[2]], a) and b.sum() == pytest.approx(a.sum())
    back = cuda.empty_like(da)
    lib.copyUnPad3DAsync(ptr(back), I(size[0]), I(size[1]), I(size[2]), ptr(big), I(logic[0]), I(logic[1]),
                         I(logic[2]), I(3), None)
    assert np.array_equal(host(cuda, back), a)


@pytest.mark.parametrize("pbc", [(0, 0, 0), (1, 1, 0)])
def test_heat_kernels(lib, cuda, pbc):
    T = rnd(SIZE, 14, 250.0, 900.0)
    k = rnd(SIZE, 15, 0.5, 1.5)
    Tl = rnd(SIZE, 16, 250.0, 400.0)
    dT, dk, dTl = dev(cuda, T), dev(cuda, k), dev(cuda, Tl)
    Q = cuda.empty_like(dT)
    lib.Qspat_async(ptr(Q), ptr(dT), ptr(dk), D(90.0), I(SIZE[0]), I(SIZE[1]), I(SIZE[2]), D(CS[0]), D(CS[1]),
                    D(CS[2]), I(pbc[0]), I(pbc[1]), I(pbc[2]), None)
    assert rel_err(host(cuda, Q), fields.qspat(T, k, 90.0, CS, pbc)) < 1e-12
    lib.QinterAsync(ptr(Q), ptr(dT), ptr(dTl), None, D(6e17), I(N), None)
    assert rel_err(host(cuda, Q), fields.qinter(T, Tl, None, 6e17)) < 1e-14
    C = T.copy()
    C[0, 0, 0] = 0.0
    dC = dev(cuda, C)
    lib.divAsync(ptr(Q), ptr(dT), ptr(dC), None, I(N))
    assert rel_err(host(cuda, Q), fields.div_zero(T, C)) < 1e-15


def test_add_family(lib, cuda):
    a, b, c = rnd(N, 20), rnd(N, 21), rnd(N, 22)
    da, db, dc = dev(cuda, a), dev(cuda, b), dev(cuda, c)
    out = cuda.empty_like(da)
    lib.addAsync(ptr(out), ptr(da), ptr(db), None, I(N))
    assert np.allclose(host(cuda, out), a + b, rtol=0, atol=1e-15)
    lib.maddAsync(ptr(out), ptr(da), ptr(db), D(0.3), None, I(N))
    assert np.allclose(host(cuda, out), a + 0.3 * b, rtol=0, atol=1e-15)
    lib.maddAsync(ptr(out), ptr(da), None, D(0.3), None, I(N))
    assert np.allclose(host(cuda, out), a + 0.3, rtol=0, atol=1e-15)
    lib.addMaddAsync(ptr(out), ptr(da), ptr(db), ptr(dc), D(0.7), None, I(N))
    assert np.allclose(host(cuda, out), a + 0.7 * (b + c), rtol=0, atol=1e-15)
    lib.linearCombination2Async(ptr(out), ptr(da), D(2.0), ptr(db), D(-3.0), None, I(N))
    assert np.allclose(host(cuda, out), 2 * a - 3 * b, rtol=0, atol=1e-14)
    lib.linearCombination3Async(ptr(out), ptr(da), D(2.0), ptr(db), D(-3.0), ptr(dc), D(0.5), None, I(N))
    assert np.allclose(host(cuda, out), 2 * a - 3 * b + 0.5 * c, rtol=0, atol=1e-14)
    x = dev(cuda, a)
    lib.madd2Async(ptr(x), ptr(db), D(0.5), ptr(dc), D(-0.25), None, I(N))
    assert np.allclose(host(cuda, x), a + 0.5 * b - 0.25 * c, rtol=0, atol=1e-15)
    x = dev(cuda, a)
    lib.madd1Async(ptr(x), None, D(0.5), None, I(N))
    assert np.allclose(host(cuda, x), a + 0.5, rtol=0, atol=1e-15)
    v = [dev(cuda, rnd(N, 30 + i)) for i in range(9)]
    lib.vecMaddAsync(*[ptr(t) for t in v[:3]], *[ptr(t) for t in v[3:6]], *[ptr(t) for t in v[6:9]], D(1.5), D(2.5),
                     D(3.5), None, I(N))
    for i, mul in enumerate((1.5, 2.5, 3.5)):
        assert np.allclose(host(cuda, v[i]), rnd(N, 33 + i) + mul * rnd(N, 36 + i), rtol=0, atol=1e-14)
    # complex madd (add.cu cmaddKern)
    src = dev(cuda, rnd(2 * N, 40))
    dst = dev(cuda, rnd(2 * N, 41))
    kern = dev(cuda, rnd(N, 42))
    lib.cmaddAsync(ptr(dst), D(0.3), D(-0.7), ptr(kern), ptr(src), None, I(N))
    s = rnd(2 * N, 40).reshape(N, 2)
    d0 = rnd(2 * N, 41).reshape(N, 2)
    kk = rnd(N, 42)
    want = d0 + np.stack([kk * (0.3 * s[:, 0] + 0.7 * s[:, 1]), kk * (-0.7 * s[:, 0] + 0.3 * s[:, 1])], 1)
    assert np.allclose(host(cuda, dst).reshape(N, 2), want, rtol=0, atol=1e-14)


def test_dots_and_partial_reductions(lib, cuda):
    A = [rnd(N, 50 + i) for i in range(6)]
    dA = [dev(cuda, a) for a in A]
    out = dev(cuda, np.zeros(N))
    lib.dotAsync(ptr(out), *[ptr(t) for t in dA], None, I(N))
    assert np.allclose(host(cuda, out), A[0] * A[3] + A[1] * A[4] + A[2] * A[5], rtol=0, atol=1e-15)
    lib.dotMaskAsync(ptr(out), *[ptr(t) for t in dA[:3]], None, None, None, D(2), D(3), D(4), D(0.5), D(0.5), D(0.5),
                     None, I(N))
    assert np.allclose(host(cuda, out), 0.5 * (2 * A[0] + 3 * A[1] + 4 * A[2]), rtol=0, atol=1e-14)
    blocks = 7
    part = dev(cuda, np.zeros(blocks))
    a, b = A[0], A[1]
    checks = [
        ("partialSumAsync", (ptr(dA[0]),), lambda p: p.sum(), a.sum()),
        ("partialSDotAsync", (ptr(dA[0]), ptr(dA[1])), lambda p: p.sum(), (a * b).sum()),
        ("partialMaxAsync", (ptr(dA[0]),), lambda p: p.max(), a.max()),
        ("partialMinAsync", (ptr(dA[0]),), lambda p: p.min(), a.min()),
        ("partialMaxAbsAsync", (ptr(dA[0]),), lambda p: p.max(), np.abs(a).max()),
        ("partialMaxDiffAsync", (ptr(dA[0]), ptr(dA[1])), lambda p: p.max(), np.abs(a - b).max()),
        ("partialMaxSumAsync", (ptr(dA[0]), ptr(dA[1])), lambda p: p.max(), np.abs(a + b).max()),
        ("partialMaxNorm3SqAsync", tuple(ptr(t) for t in dA[:3]), lambda p: p.max(),
         (A[0] ** 2 + A[1] ** 2 + A[2] ** 2).max()),
        ("partialMaxNorm3SqDiffAsync", tuple(ptr(t) for t in dA), lambda p: p.max(),
         ((A[0] - A[3]) ** 2 + (A[1] - A[4]) ** 2 + (A[2] - A[5]) ** 2).max()),
    ]
    for name, ins, fin, want in checks:
        getattr(lib, name)(*ins, ptr(part), I(blocks), I(256), I(N), None)
        assert fin(host(cuda, part)) == pytest.approx(want, rel=1e-13, abs=1e-13), name


def test_exchange_golden_through_dropin(lib, cuda):
    """The reference golden hex_ref.dump pins the pre-squaring kernel; the drop-in follows
    the current kernel, which equals the oracle with squared weights."""
    from tests.golden.make_golden import CELL_PROGRAM, MU0_PY, N as NG, exchange_inputs
    msk, lex, m = exchange_inputs()
    lex0 = math.sqrt(2 * 1.3e-11 / (MU0_PY * 800e3 * 800e3))
    dm, dl = dev(cuda, m), dev(cuda, lex)
    dh = cuda.empty_like(dm)
    c = [lex0 ** 2 / (x * x) for x in CELL_PROGRAM]
    lib.exchange6Async(*comps(dh), *comps(dm), None, ptr(dl), I(NG), I(NG), I(NG), I(0), I(0), I(0), D(800e3), D(c[0]),
                       D(c[1]), D(c[2]), None)
    want = fields.exchange6(m, lex, 800e3, lex0, CELL_PROGRAM, (0, 0, 0), weight_power=2)
    assert rel_err(host(cuda, dh), want) < 1e-12


def test_remaining_mfa_kernels(lib, cuda):
    """Debye heat capacity, spin temperature, weighted temperature average, energy flow."""
    rng = np.random.default_rng(21)
    T = rng.uniform(1.0, 900.0, size=SIZE)
    T[0, 0, 0] = 1.0            # low-temperature limit branch
    Td = rng.uniform(200.0, 400.0, size=SIZE)
    Td[0, 0, 1] = 0.0
    n = rng.uniform(0.5, 2.0, size=SIZE)
    dT, dTd, dn = dev(cuda, T), dev(cuda, Td), dev(cuda, n)
    out = cuda.empty_like(dT)
    lib.cpAsync(ptr(out), ptr(dT), ptr(dTd), ptr(dn), D(1.0), I(N), None)
    assert rel_err(host(cuda, out), fields.debye_cp(T, Td, n, 1.0)) < 1e-12

    ms0 = rng.uniform(5e5, 1e6, size=SIZE)
    ms = ms0 * rng.uniform(0.05, 0.99, size=SIZE)
    ms[1, 0, 0] = 0.0
    ms[1, 0, 1] = ms0[1, 0, 1]
    dms, dms0 = dev(cuda, ms), dev(cuda, ms0)
    for S in (0.5, 3.5):
        lib.tsAsync(ptr(out), ptr(dms), ptr(dms0), None, None, D(1.0), D(1.0), D(630.0), D(S), I(N), None)
        want = fields.spin_temperature(ms, ms0, None, None, 1.0, 1.0, 630.0, S, SIZE)
        assert rel_err(host(cuda, out), want) < 1e-7

    a, b = rng.uniform(300, 900, size=SIZE), rng.uniform(300, 400, size=SIZE)
    w0, w1 = rng.uniform(0, 2, size=SIZE), rng.uniform(0, 2, size=SIZE)
    w0[2, 2, 2] = w1[2, 2, 2] = 0.0
    da, db, dw0, dw1 = dev(cuda, a), dev(cuda, b), dev(cuda, w0), dev(cuda, w1)
    lib.wavgAsync(ptr(out), ptr(da), ptr(db), ptr(dw0), ptr(dw1), None, D(1.5), D(0.7), D(0.3), None, I(N))
    assert rel_err(host(cuda, out), fields.weighted_avg(a, b, w0, w1, None, 1.5, 0.7, 0.3)) < 1e-13

    m, R = unit(22), rng.normal(size=(3,) + SIZE)
    Tc = rng.uniform(500, 700, size=SIZE)
    Tc[3, 3, 3] = 0.0
    dm, dR, dTc = dev(cuda, m), dev(cuda, R), dev(cuda, Tc)
    lib.energyFlowAsync(ptr(out), *comps(dm), *comps(dR), ptr(dTc), None, ptr(dn), D(0.5), I(N), None)
    assert rel_err(host(cuda, out), fields.energy_flow(m, R, Tc, None, n, 0.5)) < 1e-13


@pytest.mark.parametrize("pbc", [(0, 0, 0), (1, 1, 0), (0, 1, 1)])
def test_nonlocal_damping(lib, cuda, pbc):
    rng = np.random.default_rng(23)
    h = rng.normal(size=(3,) + SIZE) * 1e5
    lam = [rng.uniform(0.1, 1.0, size=SIZE) for _ in range(3)]
    lam[1][2, 3, 4] = 0.0
    ms0 = rng.uniform(0.5, 1.0, size=SIZE)
    ms0[0, 0, 0] = 0.0
    dh, dms0 = dev(cuda, h), dev(cuda, ms0)
    dl = [dev(cuda, x) for x in lam]
    out = cuda.empty_like(dh)
    lib.llbar_nonlocal00nc_async(*comps(out), *comps(dh), ptr(dms0), *[ptr(x) for x in dl], D(1e-18), D(2e-18),
                                 D(3e-18), I(SIZE[0]), I(SIZE[1]), I(SIZE[2]), D(CS[0]), D(CS[1]), D(CS[2]),
                                 I(pbc[0]), I(pbc[1]), I(pbc[2]), None)
    want = fields.llbar_nonlocal00nc(h, ms0, lam, (1e-18, 2e-18, 3e-18), CS, pbc)
    assert rel_err(host(cuda, out), want) < 1e-12
