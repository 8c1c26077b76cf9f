"""The FP64 Newell demag tensor option (no reference counterpart: hotspin computes only
Kernel_Arne, modules/kernel_magnetostatic.go:25-241).

The device arithmetic (hotspin_b200/csrc/hsb_newell.cuh, built here as host code) is checked
against the oracle's independent restatement (oracle/newell.py), its accuracy across the
near/far-field switch against extended precision, and its difference from Kernel_Arne (the
oracle's C restatement) is measured and bounded: that difference is Kernel_Arne's quadrature
error, and it is what switching a simulation to Newell changes.
"""
import ctypes
import math

import numpy as np
import pytest

from oracle import demag, native
from oracle import newell as N

D3 = ctypes.c_double * 3


@pytest.fixture(scope="module")
def lib(host_rules):
    host_rules.newell_host.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    host_rules.newell_host.restype = None
    host_rules.newell_kernel_host.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    host_rules.newell_kernel_host.restype = None
    return host_rules


def _dev(lib, pair, R, cs):
    out = D3()
    lib.newell_host(pair[0], pair[1], D3(*R), D3(*cs), out)
    return out[0], out[1], out[2]


def test_device_arithmetic_matches_the_oracle(lib):
    rng = np.random.default_rng(7)
    for _ in range(300):
        cs = tuple(float(v) for v in rng.uniform(1.0, 4.0, 3))
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        R = tuple(float(v) for v in d * rng.uniform(0.0, 30.0) * max(cs))
        dist = np.linalg.norm(R) / max(cs)
        # the near-field differences lose ~(R/a)^5 of the FP64 digits: two implementations of
        # them agree to that level (the accuracy itself is checked against extended precision)
        tol = 1e-12 if dist < 2 else (1e-10 if dist < 5 else 1e-7)
        for pair in N.PAIRS:
            ex, asy, chosen = _dev(lib, pair, R, cs)
            want_ex = float(N.newell_exact(pair, R, cs))
            scale = max(abs(float(N.newell_exact((0, 0), R, cs))), abs(want_ex), 1e-300)
            if dist < N.NEWELL_CUTOFF:
                assert abs(ex - want_ex) <= tol * scale
            if dist > 2:
                want_as = N.newell_asymptotic(pair, R, cs)
                assert abs(asy - want_as) <= 1e-12 * max(abs(want_as), scale)
            assert chosen == (ex if dist < N.NEWELL_CUTOFF else asy)


def test_self_terms_and_trace():
    # N of a cell on itself: 1/3 each for a cube; trace 1 for any box
    for cs in ((1.0, 1.0, 1.0), (1.0, 2.0, 3.0), (5.0, 2.5, 1.0)):
        diag = [float(N.newell_exact((i, i), (0.0, 0.0, 0.0), cs)) for i in range(3)]
        assert sum(diag) == pytest.approx(1.0, abs=1e-13)
        if cs[0] == cs[1] == cs[2]:
            assert diag == pytest.approx([1 / 3] * 3, abs=1e-14)


@pytest.mark.parametrize("cs", [(1.0, 1.0, 1.0), (2.0, 1.0, 1.0), (1.0, 4.0, 4.0), (1.0, 2.0, 3.0)])
def test_switch_keeps_fp64_accuracy(lib, cs):
    """Across the near/far-field switch the tensor stays within 1e-7 of the largest entry at
    that offset, measured against the near-field formula in extended precision."""
    rng = np.random.default_rng(11)
    for dist in (6.0, 9.0, 10.9, 11.1, 14.0, 20.0):
        for _ in range(4):
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            R = tuple(float(v) for v in d * dist * max(cs))
            ref = {p: float(N.newell_exact(p, R, cs, dtype=np.longdouble)) for p in N.PAIRS}
            scale = max(abs(v) for v in ref.values())
            for p in N.PAIRS:
                _, _, got = _dev(lib, p, R, cs)
                assert abs(got - ref[p]) <= 1e-7 * scale, (cs, dist, p)


CASES = [((1, 8, 16), (3e-9, 3.9e-9, 3.9e-9), (0, 0, 0)), ((4, 8, 8), (2e-9, 2e-9, 2e-9), (0, 0, 0)),
         ((2, 8, 16), (5e-9, 2.5e-9, 1e-9), (0, 0, 0)), ((1, 16, 16), (2e-9, 2e-9, 2e-9), (0, 2, 2))]


@pytest.mark.parametrize("size,cs,pbc", CASES)
def test_folded_kernel_matches_oracle_and_stays_near_arne(lib, size, cs, pbc):
    logic = demag.pad_size(size, pbc)
    h = [l // 2 for l in logic]
    Kn = np.zeros((6, h[0] + 1, h[1] + 1, h[2] + 1))
    lib.newell_kernel_host((ctypes.c_int * 3)(*logic), (ctypes.c_int * 3)(*pbc), D3(*cs),
                           Kn.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    want = N.newell_kernel(logic, cs, pbc)
    scale = np.abs(want[:3]).max()
    assert np.abs(Kn - want).max() <= 1e-12 * scale
    Ka = native.kernel_arne(logic, cs, pbc, 6)[:, :h[0] + 1, :h[1] + 1, :h[2] + 1]
    diff = np.abs(Kn - Ka).max() / scale
    print("\n[newell vs Kernel_Arne] size %s cells %s pbc %s: max |K_newell - K_arne| = %.1e of max |K_ii|"
          % (size, cs, pbc, diff))
    assert diff < 2e-3


@pytest.mark.parametrize("size,cs,pbc", CASES)
def test_arne_quadrature_split_over_lanes_matches_oracle(host_rules, size, cs, pbc):
    """k_arne_kernel splits each target's quadrature over the 32 lanes of a warp; the shares,
    summed, equal the oracle's sequential Kernel_Arne (oracle/csrc, the reference's order) to
    rounding."""
    f = host_rules.arne_kernel_host
    f.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                  ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    f.restype = None
    logic = demag.pad_size(size, pbc)
    h = [l // 2 for l in logic]
    want = native.kernel_arne(logic, cs, pbc, 6)[:, :h[0] + 1, :h[1] + 1, :h[2] + 1]
    scale = np.abs(want[:3]).max()
    for nparts in (1, 32):
        K = np.zeros((6, h[0] + 1, h[1] + 1, h[2] + 1))
        f((ctypes.c_int * 3)(*logic), (ctypes.c_int * 3)(*pbc), D3(*cs), 6, nparts,
          K.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        # a different order of summation over up to 31104 points of cancelling contributions
        assert np.abs(K - want).max() <= (0.0 if nparts == 1 else 1e-12) * scale, nparts
