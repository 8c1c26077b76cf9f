"""Hand-written FP32 FFT demag convolution and FP64 GPU Kernel_Arne against the oracle."""
import ctypes
import os

import numpy as np
import pytest

from hotspin_b200 import _lib
from hotspin_b200.sim import demag_plan
from oracle import demag, native
from tests.gpu_util import dev, host, ptr, rel_err

pytestmark = pytest.mark.gpu

GEOMS = [
    # (size program order, cellsize, pbc)
    ((1, 32, 128), (3e-9, 3.90625e-9, 3.90625e-9), (0, 0, 0)),    # thin film, fused yz (L0 = 1)
    ((4, 32, 64), (4e-9, 4e-9, 4e-9), (0, 0, 0)),                  # fused, L0 = 8 (direct z)
    ((2, 16, 32), (2e-9, 3e-9, 4e-9), (0, 0, 0)),                  # fused, L0 = 4 (direct z)
    ((8, 16, 32), (2e-9, 2e-9, 2e-9), (0, 0, 0)),                  # fused, L0 = 16
    ((16, 16, 16), (1e-9, 2.5e-9, 5e-9), (0, 0, 0)),               # multipass (L0 = 32)
    ((16, 1024, 4), (2e-9, 2e-9, 2e-9), (0, 0, 0)),                # multipass, 2048-point y split
    ((64, 8, 8), (1e-9, 2e-9, 2e-9), (0, 0, 0)),                   # multipass, z length 128
    ((32, 8, 16), (2e-9, 3e-9, 2e-9), (1, 0, 0)),                  # multipass, periodic z (L0 = N0 = 32)
    ((4, 8, 16), (1e-9, 2e-9, 3e-9), (2, 0, 3)),                   # periodic axes
    ((1, 1, 64), (2e-9, 2e-9, 2e-9), (0, 0, 0)),                   # a single row
    ((1, 8, 2048), (2e-9, 2e-9, 2e-9), (0, 0, 0)),                 # x length 4096 (2048-point rows)
]


def _kernel_host(plan, logic):
    C2 = logic[2] // 2 + 1
    cnt = C2 * (logic[1] // 2 + 1) * (logic[0] // 2 + 1) * 6
    buf = np.empty(cnt, dtype=np.float32)
    lib = _lib.load()
    _lib.check(lib.hsb_demag_kernel_copy(plan, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), cnt))
    # [kx][k1][k0][6] -> (6, k0, k1, kx)
    return buf.reshape(C2, logic[1] // 2 + 1, logic[0] // 2 + 1, 6).transpose(3, 2, 1, 0)


@pytest.mark.parametrize("size,cs,pbc", GEOMS)
def test_kernel_spectrum_matches_oracle(cuda, size, cs, pbc):
    logic = demag.pad_size(size, pbc)
    plan = demag_plan(size, cs, pbc)
    try:
        got = _kernel_host(plan, logic)
        want = demag.kernel_spectrum(native.kernel_arne(logic, cs, pbc))
        assert got.shape == want.shape
        assert rel_err(got, want) < 2e-6
        info = (ctypes.c_double)()
        _lib.check(_lib.load().hsb_demag_plan_info(plan, None, None, ctypes.byref(info)))
        assert info.value < 1e-9   # imaginary part of the folded kernel (the reference allows 1e-12 relative)
    finally:
        _lib.load().hsb_demag_plan_destroy(plan)


@pytest.mark.parametrize("size,cs,pbc", GEOMS)
def test_demag_field_matches_oracle(cuda, size, cs, pbc):
    rng = np.random.default_rng(3)
    m = rng.normal(size=(3,) + size)
    m /= np.sqrt((m * m).sum(0))
    mask = rng.uniform(0.2, 1.0, size=size)
    logic = demag.pad_size(size, pbc)
    Kf = demag.kernel_spectrum(native.kernel_arne(logic, cs, pbc))
    want = demag.demag_field(m, mask, 8e5, Kf, logic) / demag.MU0     # A/m
    plan = demag_plan(size, cs, pbc)
    try:
        dm = dev(cuda, m, np.float32)
        dk = dev(cuda, mask, np.float32)
        H = cuda.empty_like(dm)
        _lib.check(_lib.load().hsb_demag_field(plan, ptr(dm), ptr(dk), 8e5, ptr(H), None))
        got = host(cuda, H)
        assert rel_err(got, want) < 2e-5
        # twice in a row: the plan's scratch must not leak state between calls
        _lib.check(_lib.load().hsb_demag_field(plan, ptr(dm), None, 8e5, ptr(H), None))
        want2 = demag.demag_field(m, None, 8e5, Kf, logic) / demag.MU0
        assert rel_err(host(cuda, H), want2) < 2e-5
    finally:
        _lib.load().hsb_demag_plan_destroy(plan)


def test_demag_golden_64cube(cuda):
    """The reference's tests/test-demag goldens through the FP32 GPU path."""
    from tests.golden.make_golden import CELL_PROGRAM, N, demag_inputs
    gold = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_subsample.npz"))
    sample = gold["sample_flat_index"]
    msk, m = demag_inputs()
    for tag, pbc in (("", (0, 0, 0)), ("_pbc", (2, 4, 8))):
        plan = demag_plan((N, N, N), CELL_PROGRAM, pbc)
        try:
            dm = dev(cuda, m, np.float32)
            dk = dev(cuda, msk, np.float32)
            H = cuda.empty_like(dm)
            _lib.check(_lib.load().hsb_demag_field(plan, ptr(dm), ptr(dk), 800e3, ptr(H), None))
            B = host(cuda, H).astype(np.float64) * demag.MU0
            ref = gold["B_ref%s" % tag]
            got = B.reshape(3, -1)[:, sample]
            assert rel_err(got, ref) < 1e-5
            assert np.abs(got - ref).sum(0).mean() < 1e-6   # the reference test's criterion
        finally:
            _lib.load().hsb_demag_plan_destroy(plan)


def test_unsupported_size_is_rejected(cuda):
    with pytest.raises(_lib.HsbError):
        demag_plan((3, 5, 6), (1e-9,) * 3, (1, 1, 1))


@pytest.mark.parametrize("size,cs,pbc", [((3, 12, 20), (2e-9, 3e-9, 4e-9), (0, 0, 0)),
                                         ((1, 25, 100), (3e-9, 5e-9, 5e-9), (0, 0, 0)),
                                         ((4, 12, 16), (2e-9, 2e-9, 2e-9), (2, 0, 0))])
def test_demag_on_grids_that_do_not_pad_to_powers_of_two(cuda, size, cs, pbc):
    """Open axes whose padded size 2N is not a power of two (the reference's cuFFT takes any
    size): the plan embeds the grid in the next power-of-two grid, and the field equals the
    oracle's convolution padded to 2N as the reference pads it."""
    rng = np.random.default_rng(8)
    m = rng.normal(size=(3,) + size)
    m /= np.sqrt((m * m).sum(0))
    mask = rng.uniform(0.2, 1.0, size=size)
    logic = demag.pad_size(size, pbc)
    Kf = demag.kernel_spectrum(native.kernel_arne(logic, cs, pbc))
    want = demag.demag_field(m, mask, 8e5, Kf, logic) / demag.MU0
    plan = demag_plan(size, cs, pbc)
    try:
        dm = dev(cuda, m, np.float32)
        dk = dev(cuda, mask, np.float32)
        H = cuda.empty_like(dm)
        _lib.check(_lib.load().hsb_demag_field(plan, ptr(dm), ptr(dk), 8e5, ptr(H), None))
        assert rel_err(host(cuda, H), want) < 2e-5
        _lib.check(_lib.load().hsb_demag_field(plan, ptr(dm), None, 8e5, ptr(H), None))
        want2 = demag.demag_field(m, None, 8e5, Kf, logic) / demag.MU0
        assert rel_err(host(cuda, H), want2) < 2e-5
    finally:
        _lib.load().hsb_demag_plan_destroy(plan)
