"""The four-step register FFT of the demag kernels (fft4, hotspin_b200/csrc/hsb_fft4.cuh), built
for the host, against NumPy's FFT.

tests/native/rule_check.cu runs fft4's two halves for every lane of a sequence in turn (the
first half of each lane writes the shared slot, then each lane's second half reads it back), as
the warp does between its two __syncwarp calls, with the kernels' lane layout of inputs
(x[B n1 + t] in lane t) and outputs (fft4_out_index).  Every length the kernels instantiate,
both directions, zero-padded inputs (ZIN) and half outputs (HOUT).
"""
import ctypes

import numpy as np
import pytest

LENGTHS = [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048]


@pytest.fixture(scope="module")
def fft4(host_rules):
    f = host_rules.fft4_host
    fp = ctypes.POINTER(ctypes.c_float)
    f.argtypes = [ctypes.c_int] * 4 + [fp, fp, fp]
    f.restype = ctypes.c_int
    host_rules.fft4_lanes.argtypes = [ctypes.c_int]
    host_rules.fft4_lanes.restype = ctypes.c_int
    return f, host_rules.fft4_lanes


def twiddles(L, B):
    """The plan's four-step twiddle matrix tw4[k1 B + n2] = exp(-2 pi i (n2 k1 mod L) / L)."""
    A = L // B
    k1, n2 = np.meshgrid(np.arange(A), np.arange(B), indexing="ij")
    a = -2.0 * np.pi * ((n2 * k1) % L) / L
    tw = np.stack([np.cos(a), np.sin(a)], axis=-1).astype(np.float32)
    return np.ascontiguousarray(tw.reshape(-1))


@pytest.mark.parametrize("L", LENGTHS)
def test_fft4_matches_numpy(fft4, L):
    f, lanes = fft4
    B = lanes(L)
    assert B >= 1 and L % B == 0 and L // B >= B and B <= 32
    tw = twiddles(L, B)
    P = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    rng = np.random.default_rng(L)
    for direction in (-1, 1):
        for zin in (0, 1):
            for hout in (0, 1):
                z = rng.normal(size=L) + 1j * rng.normal(size=L)
                if zin:
                    z[L // 2:] = 0.0
                x = np.ascontiguousarray(np.stack([z.real, z.imag], -1).astype(np.float32).reshape(-1))
                X = np.zeros(2 * L, np.float32)
                assert f(L, direction, zin, hout, P(x), P(tw), P(X)) == 0
                got = X[0::2].astype(np.float64) + 1j * X[1::2]
                z32 = x[0::2].astype(np.float64) + 1j * x[1::2]
                want = np.fft.fft(z32) if direction < 0 else np.fft.ifft(z32) * L
                keep = slice(0, L // 2) if hout and L > 1 else slice(0, L)
                err = np.abs(got[keep] - want[keep]).max() / np.abs(want).max()
                assert err < 1e-7 * max(2, int(np.log2(L))), (L, direction, zin, hout, err)
