"""FP64 restatement of hotspin's demag kernel and convolution (test infrastructure).

* ``kernel_arne`` follows ``Kernel_Arne`` (src/hotspin-core/modules/kernel_magnetostatic.go:25-241):
  brute-force integration of the field of the two charged faces of a source cell over
  a destination cell, integration density set by the distance (``accuracy``), summed over
  periodic images, then mirrored with the tensor's parities.
* ``kernel_spectrum`` follows ``MaxwellPlan.LoadKernel`` + ``extract``
  (maxwell_convolution.go:135-223, 350-388): forward FFT of each component over the logic
  size, real part of the folded quadrant, scaled 1/(L0 L1 L2).
* ``demag_field`` follows ``MaxwellPlan.UpdateB`` (maxwell_convolution.go:103-131) with the
  spectral multiply of ``tensSYMMVecMulKern`` (mul.cu:31-90); cuFFT (D2Z/Z2D, unnormalised)
  is restated with numpy's real FFTs.
"""
import math

import numpy as np

from .fields import MU0

# Tensor component order (common/index.go:23-28).
XX, YY, ZZ, YZ, XZ, XY = range(6)
_FULL = [[XX, XY, XZ], [XY, YY, YZ], [XZ, YZ, ZZ]]
# Parity of each component under a sign flip of one axis (kernel_magnetostatic.go:185-230).
_PARITY = {0: [1, 1, 1, 1, -1, -1],    # flip program X: XY, XZ odd
           1: [1, 1, 1, -1, 1, -1],    # flip program Y: XY, YZ odd
           2: [1, 1, 1, -1, -1, 1]}    # flip program Z: XZ, YZ odd


def pad_size(size, pbc):
    """engine/zeropad.go:12-22: double each non-periodic dimension larger than one."""
    return [2 * s if (s > 1 and p == 0) else s for s, p in zip(size, pbc)]


def kernel_ranges(size, pbc):
    """kernel_magnetostatic.go:243-256 (Go integer division truncates toward zero)."""
    r1, r2 = [0, 0, 0], [0, 0, 0]
    for c in range(3):
        if pbc[c] == 0:
            h = (size[c] - 1) // 2
            r1[c], r2[c] = -h, h
        else:
            r1[c], r2[c] = -(size[c] * pbc[c] - 1), size[c] * pbc[c] - 1
    if size[2] == 1 and pbc[2] == 0:
        r2[2] = 0
    return r1, r2


def _delta(d):
    d = np.abs(d)
    return np.where(d > 0, d - 1, 0).astype(np.float64)


def _axis_points(size, lo, hi):
    a = np.arange(lo, hi + 1)
    return a[np.mod(a, size) <= size // 2]


def _integrate_group(R, cs, s, counts, chunk_elems=3_000_000):
    """Field at the destination points R (P,3) of a unit-charged source pair of faces
    normal to axis s, for one integration density ``counts`` = (nv, nw, nx, ny, nz)."""
    u, v, w = s, (s + 1) % 3, (s + 2) % 3
    nv, nw, nx, ny, nz = (int(c) for c in counts)
    charge = cs[v] * cs[w] / float(nv * nw * nx * ny * nz)
    pv = -(cs[v] / 2.0) + cs[v] / (2 * nv) + np.arange(nv) * (cs[v] / nv)
    pw = -(cs[w] / 2.0) + cs[w] / (2 * nw) + np.arange(nw) * (cs[w] / nw)
    ox = -cs[0] / 2 + cs[0] / (2 * nx) + (cs[0] / nx) * np.arange(nx)
    oy = -cs[1] / 2 + cs[1] / (2 * ny) + (cs[1] / ny) * np.arange(ny)
    oz = -cs[2] / 2 + cs[2] / (2 * nz) + (cs[2] / nz) * np.arange(nz)
    PV, PW = np.meshgrid(pv, pw, indexing="ij")
    pole = np.zeros((PV.size, 3))
    pole[:, v] = PV.ravel()
    pole[:, w] = PW.ravel()
    OX, OY, OZ = np.meshgrid(ox, oy, oz, indexing="ij")
    off = np.stack([OX.ravel(), OY.ravel(), OZ.ravel()], 1)
    sub = pole.shape[0] * off.shape[0]
    step = max(1, chunk_elems // sub)
    out = np.zeros((R.shape[0], 3))
    for c0 in range(0, R.shape[0], step):
        r = R[c0:c0 + step][:, None, None, :] + off[None, None, :, :]
        acc = np.zeros((r.shape[0], 3))
        for pu, sg in ((cs[u] / 2.0, 1.0), (-cs[u] / 2.0, -1.0)):
            p = pole.copy()
            p[:, u] = pu
            d = r - p[None, :, None, :]
            rr = np.sqrt((d * d).sum(-1))
            q = sg * charge / (4.0 * math.pi * rr * rr * rr)
            acc += (d * q[..., None]).sum((1, 2))
        out[c0:c0 + step] = acc
    return out


def kernel_arne(size, cellsize, pbc, accuracy=6):
    """Real-space demag kernel, shape (6, L0, L1, L2), components XX YY ZZ YZ XZ XY."""
    cs = np.asarray(cellsize, dtype=np.float64)
    K = np.zeros((6,) + tuple(size))
    r1, r2 = kernel_ranges(size, pbc)
    L = float(cs.min())
    px = _axis_points(size[0], r1[0], r2[0])
    py = _axis_points(size[1], r1[1], r2[1])
    pz = _axis_points(size[2], r1[2], r2[2])
    # iterate over slabs of the slowest axis to bound memory for periodic images
    for x0 in range(0, len(px), 16):
        X, Y, Z = np.meshgrid(px[x0:x0 + 16], py, pz, indexing="ij")
        X, Y, Z = X.ravel(), Y.ravel(), Z.ravel()
        d = np.sqrt((_delta(X) * cs[0]) ** 2 + (_delta(Y) * cs[1]) ** 2 + (_delta(Z) * cs[2]) ** 2)
        d[d == 0] = L
        max_size = d / float(accuracy)
        R = np.stack([X * cs[0], Y * cs[1], Z * cs[2]], 1)
        n = [(np.maximum(cs[c] / max_size, 1.0) + 0.5).astype(np.int64) for c in range(3)]
        wx, wy, wz = np.mod(X, size[0]), np.mod(Y, size[1]), np.mod(Z, size[2])
        for s in range(3):
            v, w = (s + 1) % 3, (s + 2) % 3
            keys = np.stack([n[v] * 2, n[w] * 2, n[0], n[1], n[2]], 1)
            uk, inv = np.unique(keys, axis=0, return_inverse=True)
            inv = inv.ravel()
            B = np.zeros((X.size, 3))
            for g, counts in enumerate(uk):
                sel = np.nonzero(inv == g)[0]
                B[sel] = _integrate_group(R[sel], cs, s, counts)
            for dcomp in range(s, 3):
                np.add.at(K[_FULL[s][dcomp]], (wx, wy, wz), B[:, dcomp])
    # mirror into the upper halves with the component parities
    for ax in range(3):
        nlen = size[ax]
        idx = np.arange(nlen // 2 + 1, nlen)
        if idx.size == 0:
            continue
        dst = [slice(None)] * 3
        src = [slice(None)] * 3
        dst[ax] = idx
        src[ax] = nlen - idx
        for c in range(6):
            K[c][tuple(dst)] = _PARITY[ax][c] * K[c][tuple(src)]
    return K


def kernel_spectrum(K):
    """Folded real spectrum (6, L0/2+1, L1/2+1, L2/2+1), scaled by 1/(L0 L1 L2)."""
    L = K.shape[1:]
    n = float(np.prod(L))
    out = []
    for c in range(6):
        f = np.fft.rfftn(K[c])
        out.append(f.real[:L[0] // 2 + 1, :L[1] // 2 + 1, :] / n)
    return np.stack(out)


def unfold_spectrum(Kf, logic):
    """Expand the folded kernel to the full (6, L0, L1, L2/2+1) half spectrum with the sign
    flips of tensSYMMVecMulKern (mul.cu:58-70)."""
    L0, L1 = logic[0], logic[1]
    i = np.arange(L0)
    j = np.arange(L1)
    ii = np.where(i > L0 // 2, L0 - i, i)
    jj = np.where(j > L1 // 2, L1 - j, j)
    si = np.where(i > L0 // 2, -1.0, 1.0)[:, None, None]
    sj = np.where(j > L1 // 2, -1.0, 1.0)[None, :, None]
    full = Kf[:, ii][:, :, jj]
    sgn = np.ones((6,) + full.shape[1:])
    sgn[XY] = si * sj * np.ones(full.shape[1:])
    sgn[XZ] = si * np.ones(full.shape[1:])
    sgn[YZ] = sj * np.ones(full.shape[1:])
    return full * sgn


def demag_field(m, msat0T0_mask, msat0T0_mul, Kf, logic):
    """B (tesla) = mu0 Ms0 IFFT(K~ . FFT(pad(m * msat))), cropped (maxwell_convolution.go:103-131)."""
    size = m.shape[1:]
    M = m if msat0T0_mask is None else m * msat0T0_mask[None]
    pad = [(0, logic[a] - size[a]) for a in range(3)]
    F = [np.fft.rfftn(np.pad(M[c], pad)) for c in range(3)]
    K = unfold_spectrum(Kf, logic)
    Bs = [K[XX] * F[0] + K[XY] * F[1] + K[XZ] * F[2],
          K[XY] * F[0] + K[YY] * F[1] + K[YZ] * F[2],
          K[XZ] * F[0] + K[YZ] * F[1] + K[ZZ] * F[2]]
    n = float(np.prod(logic))
    mul = msat0T0_mul * MU0
    out = [np.fft.irfftn(b, s=logic, axes=(0, 1, 2))[:size[0], :size[1], :size[2]] * n * mul for b in Bs]
    return np.stack(out)


class DemagPlan:
    """Kernel spectrum cached for one geometry (MaxwellPlan.init/EnableDemag)."""

    def __init__(self, size, cellsize, pbc, accuracy=6):
        from . import native  # the C restatement of the same algorithm (fast)
        self.size = list(size)
        self.logic = pad_size(size, pbc)
        self.Kf = kernel_spectrum(native.kernel_arne(self.logic, cellsize, pbc, accuracy))

    def field(self, m, msat0T0_mask, msat0T0_mul):
        return demag_field(m, msat0T0_mask, msat0T0_mul, self.Kf, self.logic)
