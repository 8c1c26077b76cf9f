"""Replay of hotspin's per-step call sequence on the reference's own CUDA library.

TEST AND REFERENCE-ARM INFRASTRUCTURE.  hotspin's host is Go (no toolchain in this image), so
its engine cannot run; its CUDA kernel library can (built from the reference sources by
``oracle/ref.mk`` into ``oracle/_ref/libhotspin.so``).  This module issues the calls the Go
updaters issue for one right-hand side, in their order, each followed by a stream
synchronisation as the Go code does after almost every call
(e.g. ``modules/mod_exchange6.go:59-60``):

* H_eff SumUpdater (engine/update_sum.go:29-76): zero, then vecMadd of H_ex
  (exchange6Async), B/mu0 (MaxwellPlan.UpdateB, maxwell_convolution.go:103-131: copy,
  per component zero + copyPad3D + cuFFT D2Z, tensSYMMVecMul, per component cuFFT Z2D +
  copyUnPad3D), B_ext/mu0 (scalar vecMadd), H_anis, H_lf (long_field_async), H_therm;
* llbar_torque_async, llbar_local00nc_async, llbar_RHS SumUpdater with gamma_LL;
* two-temperature model: Qspat_async, QinterAsync, the laser source (mask x pointwise value),
  Drude Ce (copy of Te), divAsync (modules/TM.go:41-59).

cuFFT is called through torch's bindings of the same library (D2Z/Z2D, unnormalised),
out of place instead of the Go plan's in-place buffer.  The Dormand-Prince step is composed
from the reference's own madd / linearCombination / partialMaxAbs / divAsync kernels (the
reference has no RK45: its solvers are euler, heun, rk12, euler-backward and am01); the thermal field's normals come from torch's CUDA
Philox generator in place of cuRAND's.  The demag kernel spectrum is computed once on the
host by the oracle's C restatement of Kernel_Arne (setup, not timed).
"""
import ctypes
import math
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libhotspin.so")

MU0 = 4.0e-7 * math.pi
KB = 1.38064881313131313e-23

D = ctypes.c_double
I = ctypes.c_int
P = ctypes.c_void_p

_SIGS = {
    "zeroArrayAsync": [P, I, P],
    "exchange6Async": [P] * 8 + [I] * 6 + [D] * 4 + [P],
    "vecMaddAsync": [P] * 9 + [D] * 3 + [P, I],
    "maddAsync": [P, P, P, D, P, I],
    "madd1Async": [P, P, D, P, I],
    "linearCombination2Async": [P, P, D, P, D, P, I],
    "linearCombination3Async": [P, P, D, P, D, P, D, P, I],
    "copyPad3DAsync": [P, I, I, I, P, I, I, I, I, P],
    "copyUnPad3DAsync": [P, I, I, I, P, I, I, I, I, P],
    "tensSYMMVecMul": [P] * 12 + [D, I, I, I, P],
    "uniaxialAnisotropyAsync": [P] * 8 + [D, P, D, P, D, P, D, P, I],
    "long_field_async": [P] * 11 + [D] * 5 + [I, P],
    "temperature_scaleAnizNoise": [P] * 8 + [D] * 4 + [P, I],
    "llbar_torque_async": [P] * 10 + [P, I],
    "llbar_local00nc_async": [P] * 10 + [D] * 3 + [P, I],
    "Qspat_async": [P, P, P, D, I, I, I, D, D, D, I, I, I, P],
    "QinterAsync": [P, P, P, P, D, I, P],
    "divAsync": [P, P, P, P, I],
    "partialMaxAbsAsync": [P, P, I, I, I, P],
    "partialMaxDiffAsync": [P, P, P, I, I, I, P],
    "madd2Async": [P, P, D, P, D, P, I],
    "addMaddAsync": [P, P, P, P, D, P, I],
    "normalizeAsync": [P, P, P, P, I],
}


def available():
    return os.path.exists(REF_LIB)


def load(path=None):
    """The kernel library the replay drives: the reference's own build (default), or any
    library exporting the same names, e.g. the product's FP64 drop-ins (libhsb200.so)."""
    lib = ctypes.CDLL(path or REF_LIB)
    for name, args in _SIGS.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = None
    return lib


class RefSim:
    """One simulation driven through the reference kernels (FP64 device arrays)."""

    def __init__(self, kw, dt, rtol=1e-5, mindt=1e-20, maxdt=1e-13, sync_each_call=True, lib_path=None):
        import torch
        from . import demag, native
        self.torch = torch
        self.lib = load(lib_path)
        self.kw = dict(kw)
        self.sync_each = sync_each_call
        self.size = tuple(kw["size"])
        self.n = int(np.prod(self.size))
        self.dt, self.rtol, self.mindt, self.maxdt = dt, rtol, mindt, maxdt
        self.t, self.steps, self.attempts, self.rejects = 0.0, 0, 0, 0
        dev = "cuda"
        f64 = torch.float64
        n = self.n
        z = lambda *s: torch.zeros(*s, dtype=f64, device=dev)
        self.ttm = bool(kw.get("ttm"))
        self.nch = 5 if self.ttm else 3
        self.y = z(self.nch, n)
        self.ys = z(self.nch, n)
        self.k = [z(self.nch, n) for _ in range(7)]
        self.err = z(self.nch, n)
        self.H, self.Hex, self.B, self.Hlf, self.Hth, self.Hani = (z(3, n) for _ in range(6))
        self.tq, self.rl = z(3, n), z(3, n)
        if self.ttm:
            self.Qe, self.Qsp, self.Qep, self.Qp, self.Ce, self.tmp = (z(n) for _ in range(6))
            self.spot = self._laser_spot()
        self.part = z(4096)
        self.stream = torch.cuda.current_stream()
        self.sh = P(self.stream.cuda_stream)
        if kw.get("demag"):
            pbc = tuple(kw.get("pbc", (0, 0, 0)))
            self.logic = demag.pad_size(self.size, pbc)
            Kf = demag.kernel_spectrum(native.kernel_arne(self.logic, kw["cellsize"], pbc, 6))
            self.kern = [torch.from_numpy(np.ascontiguousarray(Kf[c])).to(dev) for c in range(6)]
            self.pad = z(3, *self.logic)
            self.M = z(3, n)

    # ------------------------------------------------------------------ helpers
    @staticmethod
    def p(t):
        return P(t.data_ptr())

    def sync(self):
        if self.sync_each:
            self.stream.synchronize()

    def _laser_spot(self):
        kw = self.kw
        n0, n1, n2 = self.size
        sig = kw.get("laser_sigma", 0.0)
        if sig <= 0:
            g = np.ones(self.size)
        else:
            cs = kw["cellsize"]
            yy = (np.arange(n1) + 0.5 - 0.5 * n1) * cs[1]
            xx = (np.arange(n2) + 0.5 - 0.5 * n2) * cs[2]
            g = np.broadcast_to(np.exp(-(yy[:, None] ** 2 + xx[None, :] ** 2) / (2 * sig ** 2))[None], self.size)
        return self.torch.from_numpy(np.ascontiguousarray(g).reshape(-1)).to("cuda")

    def set(self, name, arr):
        a = self.torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float64)).to("cuda")
        if name == "m":
            self.y[:3] = a.reshape(3, -1)
        elif name == "Te":
            self.y[3] = a.reshape(-1)
        elif name == "Tl":
            self.y[4] = a.reshape(-1)

    def get(self, name):
        self.torch.cuda.synchronize()
        if name == "m":
            return self.y[:3].reshape((3,) + self.size).cpu().numpy()
        return self.y[{"Te": 3, "Tl": 4}[name]].reshape(self.size).cpu().numpy()

    # ------------------------------------------------------------------ one RHS
    def vmadd(self, dst, src, mul):
        L, p, n, s = self.lib, self.p, self.n, self.sh
        L.vecMaddAsync(p(dst[0]), p(dst[1]), p(dst[2]), p(dst[0]), p(dst[1]), p(dst[2]),
                       p(src[0]) if src is not None else None, p(src[1]) if src is not None else None,
                       p(src[2]) if src is not None else None, D(mul[0]), D(mul[1]), D(mul[2]), s, I(n))
        self.sync()

    def demag_B(self, m):
        """MaxwellPlan.UpdateB with msat0T0 multiplier and no mask."""
        torch, L, p, s = self.torch, self.lib, self.p, self.sh
        kw = self.kw
        self.M.copy_(m)
        self.sync()
        n0, n1, n2 = self.size
        L0, L1, L2 = self.logic
        specs = []
        for c in range(3):
            L.zeroArrayAsync(p(self.pad[c]), I(L0 * L1 * L2), s)
            L.copyPad3DAsync(p(self.pad[c]), I(L0), I(L1), I(L2), p(self.M[c]), I(n0), I(n1), I(n2), I(1), s)
            self.sync()
            specs.append(torch.view_as_real(torch.fft.rfftn(self.pad[c])).contiguous())  # cuFFT D2Z
            self.sync()
        L.tensSYMMVecMul(p(specs[0]), p(specs[1]), p(specs[2]), p(specs[0]), p(specs[1]), p(specs[2]),
                         *[p(k) for k in self.kern], D(kw["msat0T0"] * MU0), I(L0), I(L1), I(L2 // 2 + 1), s)
        self.sync()
        for c in range(3):
            r = torch.fft.irfftn(torch.view_as_complex(specs[c]), s=(L0, L1, L2), norm="forward")  # cuFFT Z2D
            r = r.contiguous()
            self.sync()
            L.copyUnPad3DAsync(p(self.B[c]), I(n0), I(n1), I(n2), p(r), I(L0), I(L1), I(L2), I(1), s)
            self.sync()

    def thermal(self, dt, Te):
        kw = self.kw
        if not kw.get("thermal"):
            return
        torch, L, p, s, n = self.torch, self.lib, self.p, self.sh, self.n
        self.Hth.normal_()  # the step's normals (cuRAND Philox in the reference, mod_brown.go:122)
        V = float(np.prod(kw["cellsize"]))
        lam = kw["alpha"]
        pre = KB * 2.0 / (MU0 * V * kw["gamma_ll"] * max(kw.get("cutoff_dt", 0.0), dt) * kw["msat0T0"])
        Tmask = Te if Te is not None else None
        Tmul = 1.0 if Te is not None else kw["temperature"]
        L.temperature_scaleAnizNoise(p(self.Hth[0]), p(self.Hth[1]), p(self.Hth[2]), None, None, None,
                                     p(Tmask) if Tmask is not None else None, None, D(lam[0]), D(lam[1]),
                                     D(lam[2]), D(pre * Tmul), s, I(n))
        self.sync()

    def rhs(self, t, y, out):
        kw = self.kw
        torch, L, p, s, n = self.torch, self.lib, self.p, self.sh, self.n
        m = y[:3]
        size = self.size
        cs = kw["cellsize"]
        pbc = kw.get("pbc", (0, 0, 0))
        # H_eff = sum of terms
        for c in range(3):
            L.zeroArrayAsync(p(self.H[c]), I(n), s)
        self.sync()
        if kw.get("lex", 0.0):
            lm2 = kw["lex"] ** 2
            L.exchange6Async(p(self.Hex[0]), p(self.Hex[1]), p(self.Hex[2]), p(m[0]), p(m[1]), p(m[2]), None, None,
                             I(size[0]), I(size[1]), I(size[2]), I(pbc[0]), I(pbc[1]), I(pbc[2]),
                             D(kw["msat0T0"]), D(lm2 / cs[0] ** 2), D(lm2 / cs[1] ** 2), D(lm2 / cs[2] ** 2), s)
            self.sync()
            self.vmadd(self.H, self.Hex, (1.0, 1.0, 1.0))
        if kw.get("demag"):
            self.demag_B(m)
            self.vmadd(self.H, self.B, (1 / MU0,) * 3)
        b = kw.get("b_ext", (0.0, 0.0, 0.0))
        self.vmadd(self.H, None, tuple(x / MU0 for x in b))
        if kw.get("ku", 0.0):
            u = kw.get("anis_u", (0, 0, 1))
            L.uniaxialAnisotropyAsync(p(self.Hani[0]), p(self.Hani[1]), p(self.Hani[2]), p(m[0]), p(m[1]), p(m[2]),
                                      None, None, D(2 * kw["ku"] / (MU0 * kw["msat0T0"])), None, D(u[0]), None,
                                      D(u[1]), None, D(u[2]), s, I(n))
            self.sync()
            self.vmadd(self.H, self.Hani, (1.0, 1.0, 1.0))
        if kw.get("llb"):
            Te = y[3] if self.ttm else None
            L.long_field_async(p(self.Hlf[0]), p(self.Hlf[1]), p(self.Hlf[2]), p(m[0]), p(m[1]), p(m[2]), None, None,
                               None, None, p(Te) if Te is not None else None, D(kw["msat0T0"]), D(kw["spin_j"]),
                               D(kw["n_spins"]), D(kw["tc"]), D(1.0 if Te is not None else kw["temperature"]),
                               I(n), s)
            self.sync()
            self.vmadd(self.H, self.Hlf, (1.0, 1.0, 1.0))
        if kw.get("thermal"):
            self.vmadd(self.H, self.Hth, (1.0, 1.0, 1.0))
        # LLBar right-hand side
        g = kw["gamma_ll"]
        lam = kw["alpha"]
        L.llbar_torque_async(p(self.tq[0]), p(self.tq[1]), p(self.tq[2]), p(m[0]), p(m[1]), p(m[2]),
                             p(self.H[0]), p(self.H[1]), p(self.H[2]), None, s, I(n))
        self.sync()
        L.llbar_local00nc_async(p(self.rl[0]), p(self.rl[1]), p(self.rl[2]), p(self.H[0]), p(self.H[1]),
                                p(self.H[2]), None, None, None, None, D(lam[0]), D(lam[1]), D(lam[2]), s, I(n))
        self.sync()
        o = out[:3]
        for c in range(3):
            L.zeroArrayAsync(p(o[c]), I(n), s)
        self.sync()
        self.vmadd(o, self.tq, (g, g, g))
        self.vmadd(o, self.rl, (g, g, g))
        if self.ttm:
            Te, Tl = y[3], y[4]
            L.Qspat_async(p(self.Qsp), p(Te), None, D(kw["k_e"]), I(size[0]), I(size[1]), I(size[2]), D(cs[0]),
                          D(cs[1]), D(cs[2]), I(pbc[0]), I(pbc[1]), I(pbc[2]), s)
            self.sync()
            L.QinterAsync(p(self.Qep), p(Te), p(Tl), None, D(kw["g_ep"]), I(n), s)
            self.sync()
            L.zeroArrayAsync(p(self.Qe), I(n), s)
            self.sync()
            L.madd1Async(p(self.Qe), p(self.Qsp), D(1.0), s, I(n))
            self.sync()
            L.madd1Async(p(self.Qe), p(self.Qep), D(1.0), s, I(n))
            self.sync()
            tt = (t - kw["laser_t0"]) / kw["laser_fwhm"]
            val = kw["laser_p0"] * math.exp(-4 * math.log(2) * tt * tt)
            L.madd1Async(p(self.Qe), p(self.spot), D(val), s, I(n))
            self.sync()
            self.Ce.copy_(Te)   # Drude: Ce = (n/Na) gamma Te, multiplier applied below
            self.sync()
            L.divAsync(p(out[3]), p(self.Qe), p(self.Ce), s, I(n))
            self.sync()
            # the rate quantity's multiplier 1/C_mul (TM.go:41-59), applied with a reference kernel
            L.linearCombination2Async(p(out[3]), p(out[3]), D(1.0 / kw["gamma_e"]), p(out[3]), D(0.0), s, I(n))
            self.sync()
            L.zeroArrayAsync(p(self.Qp), I(n), s)
            L.madd1Async(p(self.Qp), p(self.Qep), D(-1.0), s, I(n))
            self.sync()
            L.divAsync(p(out[4]), p(self.Qp), None, s, I(n))
            self.sync()
            L.linearCombination2Async(p(out[4]), p(out[4]), D(1.0 / kw["c_l"]), p(out[4]), D(0.0), s, I(n))
            self.sync()

    # ------------------------------------------------------------------ Dormand-Prince 4(5)
    A = [[], [1 / 5], [3 / 40, 9 / 40], [44 / 45, -56 / 15, 32 / 9],
         [19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729],
         [9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656],
         [35 / 384, 0.0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84]]
    C = [0, 1 / 5, 3 / 10, 4 / 5, 8 / 9, 1, 1]
    E = [71 / 57600, 0, -71 / 16695, 71 / 1920, -17253 / 339200, 22 / 525, -1 / 40]

    def _comb(self, dst, base, coefs, ks, h):
        """dst = base + h sum_j coefs[j] ks[j] with the reference's madd kernels."""
        L, p, s = self.lib, self.p, self.sh
        nn = dst.numel()
        L.maddAsync(p(dst), p(base), None, D(0.0), s, I(nn))
        for c, kj in zip(coefs, ks):
            if c != 0.0:
                L.madd1Async(p(dst), p(kj), D(h * c), s, I(nn))
        self.sync()

    def _maxdiff(self, a, b):
        """max |a - b| as gpu.Reductor.MaxDiff (reductor.go:141-154): partialMaxDiffAsync, then
        the host finishes the block maxima.  512 threads per block: at 1024 (what the Go
        reductor picks on this GPU) the kernel's first shared-memory fold reads
        sdata[tid + 256] where it needs sdata[tid + 512] (reduce.cu, _gpu_maxdiff_kernel), so
        the upper half of each block never enters the maximum."""
        L, p, s = self.lib, self.p, self.sh
        nn = a.numel()
        threads = 512
        while nn <= threads:
            threads //= 2
        blocks = (nn + 2 * threads - 1) // (2 * threads)
        if self.part.numel() < blocks:
            self.part = self.torch.zeros(blocks, dtype=self.torch.float64, device="cuda")
        L.partialMaxDiffAsync(p(a), p(b), p(self.part), I(blocks), I(threads), I(nn), s)
        self.stream.synchronize()
        return float(self.part[:blocks].max().item())

    def _normalize(self, y):
        """The normalizer module's in-place renormalisation of m (mod_normalize.go:45-55)."""
        if self.kw.get("normalize"):
            self.lib.normalizeAsync(self.p(y[0]), self.p(y[1]), self.p(y[2]), self.sh, I(self.n))
            self.sync()

    def step_rk12(self, maxerr):
        """One step of hotspin's adaptive Heun solver (solve_rk12.go:91-214) on the reference
        kernels: inputs updated (m renormalised, dy0 = f(y0)), y0 and dy0 kept; per attempt
        the Euler predictor y = y0 + dt dy0 (Madd), m renormalised by its update, dy1 at
        t0 + dt, the corrector y += dt/2 dy1 - dt/2 dy0 (madd2Async), and per equation
        err = MaxDiff(dy1, dy0) dt; the step-size rule is the oracle's restatement of
        solve_rk12.go:148-199 (oracle.solvers.rk12_rule).  maxerr: {"m": .., "Te": .., "Tl": ..},
        a missing temperature limit leaving that equation uncontrolled.  Without a thermal
        field (the reference redraws its noise at every update)."""
        from .solvers import rk12_rule
        L, p, s = self.lib, self.p, self.sh
        assert not self.kw.get("thermal")
        nn = self.nch * self.n
        if not hasattr(self, "y0b"):
            self.y0b = self.torch.zeros_like(self.y)
        keys = [("m", slice(0, 3))] + ([("Te", slice(3, 4)), ("Tl", slice(4, 5))] if self.ttm else [])
        limits = [maxerr.get(k, math.inf) for k, _ in keys]
        t0 = self.t
        self._normalize(self.y)
        dy0, dy1 = self.k[0], self.k[1]
        self.rhs(t0, self.y, dy0)
        self.y0b.copy_(self.y)
        self.sync()
        tr = 0
        while True:
            dt = self.dt
            L.maddAsync(p(self.y), p(self.y0b), p(dy0), D(dt), s, I(nn))
            self.sync()
            self._normalize(self.y)
            self.rhs(t0 + dt, self.y, dy1)
            L.madd2Async(p(self.y), p(dy1), D(0.5 * dt), p(dy0), D(-0.5 * dt), s, I(nn))
            self.sync()
            errs = [self._maxdiff(dy1[sl], dy0[sl]) * dt for _, sl in keys]
            accept, bad, newdt, _ = rk12_rule(dt, errs, limits, self.mindt, self.maxdt)
            self.attempts += 1
            self.dt = newdt
            if accept:
                break
            if tr > 10:
                raise RuntimeError("The solver cannot converge after 10 badsteps")
            self.rejects += 1
            tr += 1
        self._normalize(self.y)          # the next update of m renormalises it
        self.t = t0 + dt
        self.steps += 1

    def _am_norm(self, a, b, scale, abs_err, rel_err):
        """solve_am01.go's error of one equation on the reference's reductions: per component,
        MaxDiff(a_p, b_p) / (maxAbsError + MaxAbs(scale_p) maxRelError), root mean square."""
        t = 0.0
        for p_ in range(a.shape[0]):
            d = self._maxdiff(a[p_], b[p_])
            mx = self._maxabs(scale[p_])
            v = d / (abs_err + mx * rel_err) if (abs_err + mx * rel_err) != 0 else math.inf
            t += v * v
        return math.sqrt(t) / math.sqrt(a.shape[0])

    def step_am12(self, abs_err, rel_err):
        """One step of hotspin's adaptive Adams-Moulton 1-2 solver (solve_am01.go:45-318) on the
        reference kernels: inputs updated (m renormalised), y0 and dy0 kept; per try the
        explicit Euler start (Madd), the implicit Euler predictor and the trapezoidal corrector
        solved by fixed-point sweeps (Madd / AddMadd, MaxDiff / MaxAbs per component), the
        step error of corrector against predictor and the new dt.  The decisions follow the Go
        code as the oracle restates them (oracle.solvers.am_iter_rule); abs_err / rel_err:
        {"m": .., "Te": .., "Tl": ..}.  Without a thermal field."""
        from .solvers import am_iter_rule
        L, p, s = self.lib, self.p, self.sh
        assert not self.kw.get("thermal")
        nn = self.nch * self.n
        torch = self.torch
        keys = [("m", slice(0, 3))] + ([("Te", slice(3, 4)), ("Tl", slice(4, 5))] if self.ttm else [])
        ab = [abs_err[k] for k, _ in keys]
        rl = [rel_err[k] for k, _ in keys]
        if not hasattr(self, "y0b"):
            self.y0b = torch.zeros_like(self.y)
            self.y1b = torch.zeros_like(self.y)
        t0 = self.t
        self._normalize(self.y)
        dy0, dybuf, dy = self.k[0], self.k[1], self.k[2]
        self.rhs(t0, self.y, dy0)
        self.y0b.copy_(self.y)
        self.sync()
        tries, restrict, s_alpha = 0, False, [0.0] * len(keys)
        while True:
            dt = self.dt
            L.maddAsync(p(self.y), p(self.y0b), p(dy0), D(dt), s, I(nn))
            self.sync()
            self._normalize(self.y)
            self.rhs(t0 + dt, self.y, dy)
            dybuf.copy_(dy)
            self.sync()
            failed = False
            for phase in (0, 1):
                er = [0.1] * len(keys)
                it = 0
                while True:
                    terrs = []
                    for (k, sl) in keys:
                        if phase == 0:
                            L.maddAsync(p(self.ys[sl]), p(self.y0b[sl]), p(dy[sl]), D(dt), s,
                                        I(self.n * (sl.stop - sl.start)))
                        else:
                            L.addMaddAsync(p(self.ys[sl]), p(self.y0b[sl]), p(dy[sl]), p(dy0[sl]), D(0.5 * dt), s,
                                           I(self.n * (sl.stop - sl.start)))
                        self.sync()
                        i = [kk for kk, _ in keys].index(k)
                        terrs.append(self._am_norm(self.y[sl], self.ys[sl], self.ys[sl], ab[i], rl[i]))
                        self.y[sl].copy_(self.ys[sl])
                    er, alp, err, alpha = am_iter_rule(er, terrs)
                    if phase == 0:
                        s_alpha = alp
                    it += 1
                    if err <= 0.1:
                        break
                    if alpha >= 1.0 or it > 5:
                        failed = True
                        break
                    self._normalize(self.y)
                    self.rhs(t0 + dt, self.y, dy)
                if failed:
                    if tries == 9:
                        raise RuntimeError("The BDF iterator cannot converge")
                    self.dt = dt * math.sqrt(0.6 / alpha) if alpha > 0.6 else 0.5 * dt
                    restrict = restrict or phase == 0
                    self.attempts += 1
                    break
                if phase == 0:
                    self.y1b.copy_(self.y)
                    dy.copy_(dybuf)
                    self.sync()
            if failed:
                continue
            bad = False
            ndts = []
            for i, (k, sl) in enumerate(keys):
                terr = self._am_norm(self.y[sl], self.y1b[sl], self.y1b[sl], ab[i], rl[i])
                bad = bad or terr > 1.0
                hr = dt * math.sqrt(0.8 / terr) if terr > 0 else math.inf
                nd = hr
                if restrict:
                    nd = min(hr, dt * math.sqrt(0.6 / s_alpha[i]) if s_alpha[i] > 0 else math.inf)
                    restrict = False
                ndts.append(min(max(nd, self.mindt), self.maxdt))
            self.attempts += 1
            self.dt = min(ndts)
            if not bad or self.dt == self.mindt:
                break
            if tries > 10:
                raise RuntimeError("The solver cannot converge after 10 badsteps")
            self.rejects += 1
            tries += 1
        self._normalize(self.y)
        self.t = t0 + dt
        self.steps += 1

    def step_rk4(self):
        """One classic RK4 step composed from the reference's madd kernels, every stage point
        and the new state renormalised when the normalizer is loaded (the device's RK4; the
        reference has no RK4)."""
        L, p, s = self.lib, self.p, self.sh
        nn = self.nch * self.n
        h, t0 = self.dt, self.t
        self._normalize(self.y)
        k = self.k
        self.rhs(t0, self.y, k[0])
        for i, (c, tf) in enumerate(((0.5, 0.5), (0.5, 0.5), (1.0, 1.0))):
            L.maddAsync(p(self.ys), p(self.y), p(k[i]), D(c * h), s, I(nn))
            self.sync()
            self._normalize(self.ys)
            self.rhs(t0 + tf * h, self.ys, k[i + 1])
        for i, w in enumerate((1.0, 2.0, 2.0, 1.0)):
            L.madd1Async(p(self.y), p(k[i]), D(w * h / 6.0), s, I(nn))
        self.sync()
        self._normalize(self.y)
        self.t = t0 + h
        self.steps += 1
        self.attempts += 1

    def _maxabs(self, a):
        L, p, s = self.lib, self.p, self.sh
        nn = a.numel()
        blocks = min(4096, (nn + 2 * 512 - 1) // (2 * 512))
        L.partialMaxAbsAsync(p(a), p(self.part), I(blocks), I(512), I(nn), s)
        self.stream.synchronize()
        return float(self.part[:blocks].max().item())   # host finish, gpu/reductor.go:113-124

    def step(self):
        kw = self.kw
        y0 = self.y
        t0 = self.t
        while True:
            h = self.dt
            self.thermal(h, y0[3] if self.ttm else None)
            ks = self.k
            self.rhs(t0, y0, ks[0])
            for sidx in range(1, 7):
                self._comb(self.ys, y0, self.A[sidx], ks[:sidx], h)
                self.rhs(t0 + self.C[sidx] * h, self.ys, ks[sidx])
            # error estimate e = h sum_j E_j k_j
            L, p, s = self.lib, self.p, self.sh
            nn = self.err.numel()
            L.linearCombination2Async(p(self.err), p(ks[0]), D(h * self.E[0]), p(ks[2]), D(h * self.E[2]), s, I(nn))
            for j in (3, 4, 5, 6):
                L.madd1Async(p(self.err), p(ks[j]), D(h * self.E[j]), s, I(nn))
            self.sync()
            err = self._maxabs(self.err[:3]) / self.rtol
            if self.ttm:
                # temperatures relative to max(|T0|, |T|), the norm of the device and the oracle
                # (the reference has no DP45 to take it from)
                scale = self.torch.maximum(y0[3:].abs(), self.ys[3:].abs())
                self.err[3:] /= scale
                self.sync()
                err = max(err, self._maxabs(self.err[3:]) / self.rtol)
            self.attempts += 1
            accept = (err <= 1.0) or h <= self.mindt
            fac = 5.0 if err == 0 else 0.9 * err ** -0.2
            fac = min(max(fac, 0.2), 5.0 if accept else 1.0)
            self.dt = min(max(h * fac, self.mindt), self.maxdt)
            if accept:
                self.y, self.ys = self.ys, self.y
                self.t = t0 + h
                self.steps += 1
                return
            self.rejects += 1


def bench_reference(args):
    """bench.py --impl reference: the reference's kernels on the bench workload, exactly the
    driver's --warmup and --steps.  Nothing of the product library is loaded here: m_e(300 K)
    of the initial state comes from the oracle's FP64 Ridders solve (oracle.fields)."""
    import json

    import torch

    from . import fields
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import bench as B
    if not available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libhotspin.so not built "
                          "(make -f oracle/ref.mk needs the reference sources)"}))
        return
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    kw = B.workload()
    st0 = B.initial_state(kw, fields.equilibrium_m(300.0, kw["tc"], kw["spin_j"]))
    sim = RefSim(kw, dt=2e-16)
    for k, v in st0.items():
        sim.set(k, v)
    steps, warm = args.steps, args.warmup
    for _ in range(warm):
        sim.step()
    torch.cuda.synchronize()
    a0, r0 = sim.attempts, sim.rejects
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record()
    for _ in range(steps):
        sim.step()
    e1.record()
    e1.synchronize()
    wall = time.perf_counter() - t0
    ms = e0.elapsed_time(e1)
    ncell = sim.n
    value = ncell * steps / (ms / 1e3) / 1e6
    out = {"impl": "reference", "metric": B.METRIC, "value": round(value, 3), "unit": B.UNIT, "n_gpus": 1,
           "steps": steps, "warmup": warm, "ms_per_step": round(ms / steps, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "parallelism": "single", "config": B.run_config(kw),
           "progress": {"attempts": sim.attempts - a0, "rejected": sim.rejects - r0,
                        "sim_time_ps_at_end": round(sim.t * 1e12, 4)},
           "path": "hotspin's own CUDA kernels (libhotspin.so built from the reference sources for sm_100a) "
                   "driven by a replay of the Go updaters' call sequence with a stream sync after each call; "
                   "cuFFT FP64; DP45 composed from the reference's madd kernels",
           "cpu_baseline": {"value": round(value, 3), "unit": B.UNIT, "cores": 1, "kind": "reference",
                            "sample": "%d accepted DP45 steps of the full workload on the reference's own "
                                      "GPU kernels (the reference has no CPU implementation of this path)"
                                      % steps},
           "e2e": {"value": round(ncell * steps / wall / 1e6, 3), "unit": B.UNIT, "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
