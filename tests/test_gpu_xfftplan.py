"""The FP64 FFT plan (hsb_fft_plan_*) against NumPy.

It stands for hotspin's FFTPlanX (gpu/fftplanX.go:76-104): forward = the data block
zero-padded to the logic size, then the unnormalised real-to-complex transform in cuFFT's packed
layout (L2 + 2 doubles per row); inverse = the unnormalised complex-to-real transform, cropped
to the data block.  Shapes cover open axes (logic = 2 x data), sizes that are not powers of two
inside a power-of-two logic size, periodic axes (logic = data), single cells and rows of 4096.
"""
import ctypes

import numpy as np
import pytest

from hotspin_b200 import _lib
from tests.gpu_util import dev, host, ptr, rel_err

pytestmark = pytest.mark.gpu

CASES = [((1, 32, 128), (1, 64, 256)), ((4, 16, 32), (8, 32, 64)), ((3, 5, 7), (8, 16, 16)),
         ((16, 16, 16), (16, 16, 16)), ((1, 1, 8), (1, 1, 16)), ((2, 4, 2048), (4, 8, 4096))]


def _plan(data, logic):
    lib = _lib.load()
    h = ctypes.c_void_p()
    I3 = ctypes.c_int * 3
    _lib.check(lib.hsb_fft_plan_create(I3(*data), I3(*logic), None, ctypes.byref(h)), "hsb_fft_plan_create")
    return lib, h


@pytest.mark.parametrize("data,logic", CASES)
def test_forward_and_inverse_match_numpy(cuda, data, logic):
    lib, plan = _plan(data, logic)
    try:
        rng = np.random.default_rng(sum(data))
        x = rng.normal(size=data)
        L0, L1, L2 = logic
        pad = np.pad(x, [(0, logic[a] - data[a]) for a in range(3)])
        want = np.fft.rfftn(pad)
        dx = dev(cuda, x)
        spec = cuda.zeros((L0, L1, L2 + 2), dtype=cuda.float64, device="cuda")
        for _ in range(2):          # twice: the plan's scratch carries nothing between calls
            _lib.check(lib.hsb_fft_forward(plan, ptr(dx), ptr(spec)), "hsb_fft_forward")
            got = host(cuda, spec).view(np.complex128)
            assert got.shape == want.shape
            assert rel_err(got, want) < 1e-12
        kept = host(cuda, spec).copy()
        back = cuda.zeros(data, dtype=cuda.float64, device="cuda")
        _lib.check(lib.hsb_fft_inverse(plan, ptr(spec), ptr(back)), "hsb_fft_inverse")
        n = L0 * L1 * L2
        assert rel_err(host(cuda, back), n * x) < 1e-12
        assert np.array_equal(host(cuda, spec), kept)        # the spectrum is left unchanged
        # the inverse of a general Hermitian spectrum (a convolution's), against NumPy's C2R
        k = rng.normal(size=logic)
        prod = want * np.fft.rfftn(k)
        dp = dev(cuda, np.ascontiguousarray(prod).view(np.float64).reshape(L0, L1, L2 + 2))
        _lib.check(lib.hsb_fft_inverse(plan, ptr(dp), ptr(back)), "hsb_fft_inverse")
        ref = np.fft.irfftn(prod, s=logic, axes=(0, 1, 2))[:data[0], :data[1], :data[2]] * n
        assert rel_err(host(cuda, back), ref) < 1e-12
    finally:
        lib.hsb_fft_plan_destroy(plan)


def test_unsupported_sizes_are_refused(cuda):
    lib = _lib.load()
    h = ctypes.c_void_p()
    I3 = ctypes.c_int * 3
    for data, logic in (((4, 4, 4), (4, 4, 6)), ((4, 4, 8), (4, 4, 4)), ((1, 1, 1), (1, 1, 1)),
                        ((2, 2, 8), (2, 2, 8192))):
        assert lib.hsb_fft_plan_create(I3(*data), I3(*logic), None, ctypes.byref(h)) == 4
        assert b"hsb_fft_plan_create" in lib.hsb_last_error()
