"""Philox4x32-10 counter-based generator and Box-Muller normals (test infrastructure).

Restates the published algorithm (J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw,
"Parallel random numbers: as easy as 1, 2, 3", SC'11): ten rounds of two 32x32->64-bit
multiplies with multipliers 0xD2511F53 / 0xCD9E8D57 and Weyl key increments
0x9E3779B9 / 0xBB67AE85.  The reference draws its thermal noise from cuRAND's
PHILOX4_32_10 generator (src/hotspin-core/modules/mod_brown.go:98,122); cuRAND's
stream layout is not reproduced (parity for the thermal field is statistical).

Stream layout used by hotspin_b200 (and restated here): one Philox call per cell and
step, counter = (cell, step_lo, step_hi, 0x48535442), key = (seed_lo, seed_hi); the first
three of the four outputs become the x, y, z normals through Box-Muller on
u = (bits + 0.5) * 2^-32.
"""
import numpy as np

M0, M1 = 0xD2511F53, 0xCD9E8D57
W0, W1 = 0x9E3779B9, 0xBB67AE85
STREAM_TAG = 0x48535442
_MASK = 0xFFFFFFFF


def _mulhilo(a, b):
    p = a.astype(np.uint64) * np.uint64(b)
    return (p >> np.uint64(32)).astype(np.uint32), (p & np.uint64(_MASK)).astype(np.uint32)


def philox4x32_10(ctr, key):
    """ctr: (4, n) uint32, key: (2,) or (2, n) uint32 -> (4, n) uint32."""
    c = [np.asarray(x, dtype=np.uint32).copy() for x in ctr]
    k0 = np.asarray(key[0], dtype=np.uint64) & np.uint64(_MASK)
    k1 = np.asarray(key[1], dtype=np.uint64) & np.uint64(_MASK)
    for r in range(10):
        hi0, lo0 = _mulhilo(c[0], M0)
        hi1, lo1 = _mulhilo(c[2], M1)
        kk0 = k0.astype(np.uint32)
        kk1 = k1.astype(np.uint32)
        c = [hi1 ^ c[1] ^ kk0, lo1, hi0 ^ c[3] ^ kk1, lo0]
        k0 = (k0 + np.uint64(W0)) & np.uint64(_MASK)
        k1 = (k1 + np.uint64(W1)) & np.uint64(_MASK)
    return np.stack(c)


def uniform01(bits):
    """(bits + 0.5) / 2^32, strictly inside (0, 1)."""
    return (bits.astype(np.float64) + 0.5) * (1.0 / 4294967296.0)


def box_muller(u0, u1):
    r = np.sqrt(-2.0 * np.log(u0))
    a = 2.0 * np.pi * u1
    return r * np.cos(a), r * np.sin(a)


def thermal_normals(ncell, step, seed):
    """(3, ncell) standard normals for one step (the layout documented above)."""
    cell = np.arange(ncell, dtype=np.uint64)
    ctr = [cell.astype(np.uint32),
           np.full(ncell, step & _MASK, dtype=np.uint32),
           np.full(ncell, (step >> 32) & _MASK, dtype=np.uint32),
           np.full(ncell, STREAM_TAG, dtype=np.uint32)]
    key = (seed & _MASK, (seed >> 32) & _MASK)
    r = philox4x32_10(ctr, key)
    n0, n1 = box_muller(uniform01(r[0]), uniform01(r[1]))
    n2, _ = box_muller(uniform01(r[2]), uniform01(r[3]))
    return np.stack([n0, n1, n2])
