"""Newell demag tensor (FP64 / extended precision) -- TEST INFRASTRUCTURE ONLY.

The reference computes only Kernel_Arne (modules/kernel_magnetostatic.go:25-241); the Newell
tensor is the closed-form alternative offered for large grids.  This is the oracle for the
device version (hotspin_b200/csrc/hsb_newell.cuh):

* exact: Newell, Williams and Dunlop, J. Geophys. Res. 98 (1993) 9551, the cell-averaged
  tensor N_ij(R) as the 27-point second difference over the three axes (weights 2, -1, -1 per
  axis) of the auxiliary functions f (diagonal) and g (off-diagonal), divided by 4 pi V;
* far field: the multipole expansion of N_ij(R) = -(V / 4 pi) E[d_i d_j (1 / |R + u|)] over
  the offset u between two uniformly distributed points of source and target cell (per axis
  the difference of two uniforms, moments <u^2> = a^2/6, <u^4> = a^4/15, <u^6> = a^6/28),
  through sixth order, with the derivatives of 1/|x| from the Taylor-coefficient recurrence
  |k| |x|^2 a_k - (2|k| - 1) sum_i x_i a_{k-e_i} + (|k| - 1) sum_i a_{k-2e_i} = 0.

K = -N is the tensor in the convention of Kernel_Arne (H = K * M).  Arrays use program
order; component indices 0, 1, 2 are program axes.
"""
import math
from functools import lru_cache

import numpy as np

# tensor entries in the order of the kernel spectrum (hsb_demag.h): XX YY ZZ YZ XZ XY
PAIRS = [(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]


def _asinh_ratio(a, b2, xp):
    """asinh(a / sqrt(b2)), 0 where b2 == 0 (its coefficient vanishes there)."""
    safe = xp.where(b2 > 0, b2, 1)
    return xp.where(b2 > 0, xp.arcsinh(a / xp.sqrt(safe)), 0)


def _atan_ratio(num, den, xp):
    """atan(num / den), 0 where den == 0 (its coefficient vanishes there)."""
    safe = xp.where(den != 0, den, 1)
    return xp.where(den != 0, xp.arctan(num / safe), 0)


def newell_f(x, y, z, xp=np):
    x2, y2, z2 = x * x, y * y, z * z
    R = xp.sqrt(x2 + y2 + z2)
    return (0.5 * y * (z2 - x2) * _asinh_ratio(y, x2 + z2, xp)
            + 0.5 * z * (y2 - x2) * _asinh_ratio(z, x2 + y2, xp)
            - x * y * z * _atan_ratio(y * z, x * R, xp)
            + (2 * x2 - y2 - z2) * R / 6)


def newell_g(x, y, z, xp=np):
    x2, y2, z2 = x * x, y * y, z * z
    R = xp.sqrt(x2 + y2 + z2)
    return (x * y * z * _asinh_ratio(z, x2 + y2, xp)
            + y * (3 * z2 - y2) * _asinh_ratio(x, y2 + z2, xp) / 6
            + x * (3 * z2 - x2) * _asinh_ratio(y, x2 + z2, xp) / 6
            - z * z2 * _atan_ratio(x * y, z * R, xp) / 6
            - z * y2 * _atan_ratio(x * z, y * R, xp) / 2
            - z * x2 * _atan_ratio(y * z, x * R, xp) / 2
            - x * y * R / 3)


def _second_difference(fun, X, Y, Z, dx, dy, dz, dtype):
    w = {-1: -1.0, 0: 2.0, 1: -1.0}
    acc = 0
    for i in (-1, 0, 1):
        for j in (-1, 0, 1):
            for k in (-1, 0, 1):
                acc = acc + w[i] * w[j] * w[k] * fun(dtype(X + i * dx), dtype(Y + j * dy), dtype(Z + k * dz))
    return acc


def newell_exact(pair, R, cs, dtype=np.float64):
    """N_ij at offset R (3 floats, program order) between cells of size cs, exact formula."""
    i, j = pair
    X, Y, Z = (dtype(v) for v in R)
    a = [dtype(v) for v in cs]
    V = a[0] * a[1] * a[2]
    if i == j:
        # f is written for the xx entry: rotate so that axis i plays x
        o = [i, (i + 1) % 3, (i + 2) % 3]
        P = [(X, Y, Z)[o[0]], (X, Y, Z)[o[1]], (X, Y, Z)[o[2]]]
        d = [a[o[0]], a[o[1]], a[o[2]]]
        s = _second_difference(newell_f, *P, *d, dtype)
    else:
        k = 3 - i - j
        P = [(X, Y, Z)[i], (X, Y, Z)[j], (X, Y, Z)[k]]
        d = [a[i], a[j], a[k]]
        s = _second_difference(newell_g, *P, *d, dtype)
    return s / (4 * dtype(math.pi) * V)


@lru_cache(maxsize=None)
def _multi_indices(order):
    return [(a, b, order - a - b) for a in range(order + 1) for b in range(order + 1 - a)]


def inv_r_derivatives(x, max_order):
    """All partial derivatives d^k (1/|x|) for |k| <= max_order, as {k: value}."""
    r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2]
    a = {(0, 0, 0): 1.0 / math.sqrt(r2)}
    for n in range(1, max_order + 1):
        for k in _multi_indices(n):
            s1 = 0.0
            s2 = 0.0
            for d in range(3):
                if k[d] >= 1:
                    km = list(k)
                    km[d] -= 1
                    s1 += x[d] * a[tuple(km)]
                if k[d] >= 2:
                    km = list(k)
                    km[d] -= 2
                    s2 += a[tuple(km)]
            a[k] = ((2 * n - 1) * s1 - (n - 1) * s2) / (n * r2)
    return {k: v * math.factorial(k[0]) * math.factorial(k[1]) * math.factorial(k[2]) for k, v in a.items()}


def newell_asymptotic(pair, R, cs):
    """N_ij at offset R from the multipole expansion through sixth order in the cell size."""
    D = inv_r_derivatives(R, 8)
    i, j = pair
    e = [0, 0, 0]
    e[i] += 1
    e[j] += 1
    s2 = [c * c / 6.0 for c in cs]          # <u^2>
    m4 = [c ** 4 / 15.0 for c in cs]        # <u^4>
    m6 = [c ** 6 / 28.0 for c in cs]        # <u^6>

    def d(*add):
        k = list(e)
        for axis, p in add:
            k[axis] += p
        return D[tuple(k)]

    total = d()
    total += 0.5 * sum(s2[k] * d((k, 2)) for k in range(3))
    t4 = sum(m4[k] * d((k, 4)) for k in range(3))
    t4 += 6 * sum(s2[k] * s2[l] * d((k, 2), (l, 2)) for k in range(3) for l in range(k + 1, 3))
    total += t4 / 24.0
    t6 = sum(m6[k] * d((k, 6)) for k in range(3))
    t6 += 15 * sum(m4[k] * s2[l] * d((k, 4), (l, 2)) for k in range(3) for l in range(3) if l != k)
    t6 += 90 * s2[0] * s2[1] * s2[2] * d((0, 2), (1, 2), (2, 2))
    total += t6 / 720.0
    V = cs[0] * cs[1] * cs[2]
    return -V / (4 * math.pi) * total


def newell(pair, R, cs, cutoff=None):
    """N_ij: exact below `cutoff` (distance in units of the largest cell edge), expansion
    above (the default matches the device)."""
    if cutoff is None:
        cutoff = NEWELL_CUTOFF
    dist = math.sqrt(sum(r * r for r in R)) / max(cs)
    if dist < cutoff:
        return float(newell_exact(pair, R, cs))
    return newell_asymptotic(pair, R, cs)


# cells (largest edge) beyond which the far-field expansion replaces the exact differences
NEWELL_CUTOFF = 11.0


def newell_kernel(logic, cs, pbc=(0, 0, 0)):
    """Folded kernel K = -N on the (L0/2+1, L1/2+1, L2/2+1) octant of the logic grid, summed over
    periodic images as Kernel_Arne's loop does (oracle/demag.py conventions)."""
    L = logic
    h = [l // 2 for l in L]
    r1, r2 = [], []
    for a in range(3):
        if pbc[a] == 0:
            r1.append(-((L[a] - 1) // 2))
            r2.append((L[a] - 1) // 2)
        else:
            r1.append(-(L[a] * pbc[a] - 1))
            r2.append(L[a] * pbc[a] - 1)
    if L[2] == 1 and pbc[2] == 0:
        r2[2] = 0
    K = np.zeros((6, h[0] + 1, h[1] + 1, h[2] + 1))
    for t0 in range(h[0] + 1):
        for t1 in range(h[1] + 1):
            for t2 in range(h[2] + 1):
                t = (t0, t1, t2)
                first = []
                for a in range(3):
                    x = t[a]
                    while x - L[a] >= r1[a]:
                        x -= L[a]
                    while x < r1[a]:
                        x += L[a]
                    first.append(x)
                acc = np.zeros(6)
                for z in range(first[2], r2[2] + 1, L[2]):
                    for y in range(first[1], r2[1] + 1, L[1]):
                        for x in range(first[0], r2[0] + 1, L[0]):
                            R = (x * cs[0], y * cs[1], z * cs[2])
                            for c, p in enumerate(PAIRS):
                                acc[c] -= newell(p, R, cs)
                K[:, t0, t1, t2] = acc
    return K


def newell_kernel_full(logic, cs, pbc=(0, 0, 0)):
    """The Newell K = -N on the whole logic grid (6, L0, L1, L2), unfolded from the octant with
    the tensor's parities (diagonal entries even in every axis, K_ij odd in axes i and j), the
    layout oracle.native.kernel_arne returns."""
    Kf = newell_kernel(logic, cs, pbc)
    L = logic
    h = [l // 2 for l in L]
    out = np.zeros((6,) + tuple(L))
    for c, (i, j) in enumerate(PAIRS):
        for a0 in range(L[0]):
            f0, s0 = (a0, 1) if a0 <= h[0] else (L[0] - a0, -1)
            for a1 in range(L[1]):
                f1, s1 = (a1, 1) if a1 <= h[1] else (L[1] - a1, -1)
                for a2 in range(L[2]):
                    f2, s2 = (a2, 1) if a2 <= h[2] else (L[2] - a2, -1)
                    sign = 1
                    if i != j:
                        for axis, s in ((0, s0), (1, s1), (2, s2)):
                            if axis in (i, j):
                                sign *= s
                    out[c, a0, a1, a2] = sign * Kf[c, f0, f1, f2]
    return out
