"""FP64 restatement of hotspin's per-cell field and torque kernels (test infrastructure).

Each function follows one kernel of ``src/libhotspin`` and the Go updater that supplies its
multipliers.  Masks follow the reference convention: ``None`` means a uniform mask of 1
(``common_func.h:140-143`` getMaskUnity) and the physical value is a separate multiplier.
All arrays are program order, see the package docstring.
"""
import math

import numpy as np

# Constants: common/constants.go:16-24 (Go side) and common_func.h:30-33 (device side).
MU0 = 4.0 * math.pi * 1e-7
KB = 1.38064881313131313e-23
MUB = 9.27400968202020202e-24
GAMMA0 = 2.211e5
NA = 6.02214129272727272e23

ZERO = 1.0e-32            # common_func.h:24
LIN_RANGE = 2.0e-1        # common_func.h:26
INFINITE_SPIN = 1.0e5     # common_func.h:28
RIDDERS_EPS = 1.0e-8      # common_func.h:25


def _mask(msk, shape):
    return np.ones(shape) if msk is None else np.asarray(msk, dtype=np.float64)


def avg_geom_zero(a, b):
    """2ab/(a+b), 0 when a+b == 0 (common_func.h:147-152)."""
    s = a + b
    safe = np.where(s == 0.0, 1.0, s)
    return np.where(s == 0.0, 0.0, 2.0 * a * b / safe)


def _neighbour_index(n, periodic, direction):
    """Index of the -1 / +1 neighbour along an axis of length n.

    Open boundaries clamp (Neumann), periodic ones wrap (exchange6.cu:40-60).
    """
    idx = np.arange(n)
    if direction < 0:
        nb = idx - 1
        if periodic:
            nb = np.where(nb < 0, n + nb, nb)
        return np.maximum(nb, 0)
    nb = idx + 1
    if periodic:
        nb = np.where(nb == n, nb - n, nb)
    return np.minimum(nb, n - 1)


def laplace_weighted(f, w, inv_cs2, pbc):
    """sum_d inv_cs2[d] * [w-(f- - f) + w+(f+ - f)] with harmonic-mean weights.

    Shared by exchange6Kern (exchange6.cu:22-116, weights from lex^2) and QspatKern
    (Qspat.cu:25-100, weights from k).  ``f`` has shape (..., N0, N1, N2); ``w`` (N0, N1, N2).
    The reference evaluates ``(pre1*f1 + pre2*f2) - (pre1*f0 + pre2*f0)``; that order is kept.
    """
    out = np.zeros_like(f)
    lead = f.ndim - 3
    for ax in range(3):
        n = w.shape[ax]
        im = _neighbour_index(n, pbc[ax], -1)
        ip = _neighbour_index(n, pbc[ax], +1)
        fm = np.take(f, im, axis=lead + ax)
        fp = np.take(f, ip, axis=lead + ax)
        p1 = avg_geom_zero(w, np.take(w, im, axis=ax))
        p2 = avg_geom_zero(w, np.take(w, ip, axis=ax))
        out += inv_cs2[ax] * ((p1 * fm + p2 * fp) - (p1 * f + p2 * f))
    return out


def exchange6(m, lex_mask, msat0T0_mul, lex_mul, cellsize, pbc, weight_power=2):
    """H_ex in A/m (exchange6.cu:11-127; multipliers from mod_exchange6.go:40-61).

    H = Ms0 * sum_d (lex_mul^2 / cs_d^2) [w-(m- - m) + w+(m+ - m)],
    w = harmonic mean of the neighbours' lex_mask^2 (the current reference kernel,
    exchange6.cu:28-60).  ``weight_power=1`` selects harmonic means of lex_mask itself,
    which is what the reference's golden ``tests/test-exchange/hex_ref*.dump`` was
    generated with (an older kernel); the two agree for a uniform lex mask.
    """
    shape = m.shape[1:]
    lex = _mask(lex_mask, shape)
    inv = [lex_mul * lex_mul / (c * c) for c in cellsize]
    return msat0T0_mul * laplace_weighted(m, lex ** weight_power, inv, pbc)


def uniaxial_anisotropy(m, ku_mask, msat_mask, ku_mul, msat_mul, u_mask, u_mul):
    """H_anis (uniaxialanisotropy.cu:12-52; multiplier mod_uniaxialanisotropy.go:44-57).

    H = (2 Ku / (mu0 Ms)) (m . u_hat) u, where the projection uses the normalised u but the
    output direction is the un-normalised u (as in the reference).  Zero where Ms mask == 0.
    """
    shape = m.shape[1:]
    msat = _mask(msat_mask, shape)
    ku = _mask(ku_mask, shape)
    pre_mul = 2.0 * ku_mul / (MU0 * msat_mul)
    safe = np.where(msat == 0.0, 1.0, msat)
    pre = (pre_mul / safe) * ku
    u = np.stack([u_mul[c] * _mask(None if u_mask is None else u_mask[c], shape) for c in range(3)])
    ulen = np.sqrt((u * u).sum(0))
    uinv = np.where(ulen != 0.0, 1.0 / np.where(ulen == 0.0, 1.0, ulen), 0.0)
    mu = (m * (u * uinv)).sum(0)
    h = pre * mu * u
    return np.where(msat == 0.0, 0.0, h)


def ref_cross(a, b):
    """The reference's ``cross(a, b)`` (common_func.h:52-55), which evaluates b x a:
    x = -a.y b.z + a.z b.y, and so on."""
    return np.cross(b, a, axis=0)


def llbar_torque(m, h, msat0T0_mask, gamma_ll):
    """gamma_LL * cross(H, M) = gamma_LL * (m x H) (llbar-torque.cu:11-45 with the
    reference's cross helper, common_func.h:52-55).

    The reference kernel writes the bare cross product and sets gamma_LL as the quantity's
    multiplier (mod_llbar-torque.go:55-68); the product is applied here.  Zero in vacuum.
    """
    shape = m.shape[1:]
    ms = _mask(msat0T0_mask, shape)
    t = ref_cross(h, m)
    return np.where(ms == 0.0, 0.0, gamma_ll * t)


def llbar_local00nc(h, msat0T0_mask, lam_mask, lam_mul, gamma_ll):
    """gamma_LL * diag(lambda) H (llbar-local00nc.cu:11-63; mod_llbar-local00nc.go:77-99)."""
    shape = h.shape[1:]
    ms = _mask(msat0T0_mask, shape)
    lam = np.stack([lam_mul[c] * _mask(None if lam_mask is None else lam_mask[c], shape)
                    for c in range(3)])
    return np.where(ms == 0.0, 0.0, gamma_ll * lam * h)


def llbar_local02nc(m, h, msat0T0_mask, mu_mask, mu_mul, gamma_ll):
    """gamma_LL * diag(mu) (m.H) m (llbar-local02nc.cu:11-73)."""
    shape = h.shape[1:]
    ms = _mask(msat0T0_mask, shape)
    mu = np.stack([mu_mul[c] * _mask(None if mu_mask is None else mu_mask[c], shape)
                   for c in range(3)])
    mh = (m * h).sum(0)
    return np.where(ms == 0.0, 0.0, gamma_ll * mu * mh * m)


def llbar_local02c(m, h, msat0T0_mask, mu_mask, mu_mul, gamma_ll):
    """gamma_LL * cross(diag(mu) cross(m, H), m) with the reference's cross helper
    (llbar-local02c.cu:11-69, common_func.h:52-55)."""
    shape = h.shape[1:]
    ms = _mask(msat0T0_mask, shape)
    mu = np.stack([mu_mul[c] * _mask(None if mu_mask is None else mu_mask[c], shape)
                   for c in range(3)])
    a = mu * ref_cross(m, h)
    return np.where(ms == 0.0, 0.0, gamma_ll * ref_cross(a, m))


def normalize(m):
    """m / |m|, zero stays zero (normalize.cu:13-46)."""
    n = np.sqrt((m * m).sum(0))
    inv = np.where(n == 0.0, 0.0, 1.0 / np.where(n == 0.0, 1.0, n))
    return m * inv


# ----------------------------------------------------------------------------- MFA
def _coth(x):
    return 1.0 / np.tanh(x)


def brillouin(J, x):
    """B_J(x) with the reference's 4-term series below linRange (common_func.h:72-97)."""
    x = np.asarray(x, dtype=np.float64)
    lpre = 1.0 / (2.0 * J)
    gpre = (2.0 * J + 1.0) * lpre
    g2, l2 = gpre * gpre, lpre * lpre
    g4, l4 = g2 * g2, l2 * l2
    g6, l6 = g4 * g2, l4 * l2
    g8, l8 = g4 * g4, l4 * l4
    lim = min(LIN_RANGE / gpre, LIN_RANGE / lpre)
    small = np.abs(x) < lim
    xs = np.where(small, x, 0.0)
    ser = ((g2 - l2) * xs / 3.0 - (g4 - l4) * xs ** 3 / 45.0
           + (g6 - l6) * xs ** 5 * 2.0 / 945.0 - (g8 - l8) * xs ** 7 / 4725.0)
    xl = np.where(small, 1.0, x)
    full = gpre * _coth(gpre * xl) - lpre * _coth(lpre * xl)
    return np.where(small, ser, full)


def dbrillouin(J, x):
    """dB_J/dx (common_func.h:99-120)."""
    x = np.asarray(x, dtype=np.float64)
    lpre = 1.0 / (2.0 * J)
    gpre = (2.0 * J + 1.0) * lpre
    g2, l2 = gpre * gpre, lpre * lpre
    g4, l4 = g2 * g2, l2 * l2
    g6, l6 = g4 * g2, l4 * l2
    g8, l8 = g4 * g4, l4 * l4
    lim = min(LIN_RANGE / gpre, LIN_RANGE / lpre)
    small = np.abs(x) < lim
    xs = np.where(small, x, 0.0)
    ser = ((g2 - l2) / 3.0 - (g4 - l4) * xs ** 2 / 15.0
           + (g6 - l6) * xs ** 4 * 2.0 / 189.0 - (g8 - l8) * xs ** 6 / 675.0)
    xl = np.where(small, 1.0, x)
    cl, cg = _coth(lpre * xl), _coth(gpre * xl)
    full = (g2 - l2) + l2 * cl * cl - g2 * cg * cg
    return np.where(small, ser, full)


def langevin(x):
    """L(x) (common_func.h:122-129)."""
    x = np.asarray(x, dtype=np.float64)
    small = np.abs(x) < LIN_RANGE
    xs = np.where(small, x, 0.0)
    ser = xs / 3.0 - xs ** 3 / 45.0 + xs ** 5 * 2.0 / 945.0 - xs ** 7 / 4725.0
    xl = np.where(small, 1.0, x)
    return np.where(small, ser, _coth(xl) - 1.0 / xl)


def dlangevin(x):
    """dL/dx (common_func.h:131-138)."""
    x = np.asarray(x, dtype=np.float64)
    small = np.abs(x) < LIN_RANGE
    xs = np.where(small, x, 0.0)
    ser = 1.0 / 3.0 - xs ** 2 / 15.0 + xs ** 4 * 2.0 / 189.0 - xs ** 6 / 675.0
    xl = np.where(small, 1.0, x)
    c = _coth(xl)
    return np.where(small, ser, 1.0 - c * c + 1.0 / (xl * xl))


def long_field(m, msat0T0_mask, S_mask, n_mask, Tc_mask, T_mask,
               msat0T0_mul, S_mul, n_mul, Tc_mul, T_mul):
    """MFA longitudinal field H_lf (long_field.cu:13-72; mod_long_field.go:74-86).

    H_lf = n kB T (W(|m| b) - |m|) / (mu0 Ms0 W'(|m| b)) * m_hat, b = 3 S/(S+1) Tc/T,
    W = B_S (Langevin when S > 1e5).  Zero where Ms0 == 0, n == 0 or |m| <= 1e-32.
    """
    shape = m.shape[1:]
    ms0 = msat0T0_mul * _mask(msat0T0_mask, shape)
    S = S_mul * _mask(S_mask, shape)
    n = n_mul * _mask(n_mask, shape)
    Tc = Tc_mul * _mask(Tc_mask, shape)
    T = T_mul * _mask(T_mask, shape)
    a = np.sqrt((m * m).sum(0))
    out = np.zeros_like(m)
    ok = (ms0 != 0.0) & (n != 0.0) & (a > ZERO)
    if not ok.any():
        return out
    # Per-cell spin values may differ; evaluate per unique S (the configs use one S).
    for s in np.unique(S[ok]):
        sel = ok & (S == s)
        pre_s = 1.0 if s > INFINITE_SPIN else s / (s + 1.0)
        b = 3.0 * pre_s * Tc[sel] / T[sel]
        meb = a[sel] * b
        if s > INFINITE_SPIN:
            W, dW = langevin(meb), dlangevin(meb)
        else:
            W, dW = brillouin(s, meb), dbrillouin(s, meb)
        mult = n[sel] * KB * T[sel] * (W - a[sel]) / (MU0 * ms0[sel] * dW)
        for c in range(3):
            out[c][sel] = mult * (m[c][sel] / a[sel])
    return out


def _ridders(f, xa, xb):
    """Ridders' root bracket iteration exactly as findroot_Ridders (brillouin.cu:13-71)."""
    ya = f(xa)
    if abs(ya) < ZERO:
        return xa
    yb = f(xb)
    if abs(yb) < ZERO:
        return xb
    y1, x1, y2, x2 = ya, xa, yb, xb
    x = 1.0e10
    tx = x
    teps = x
    it = 0
    while teps > RIDDERS_EPS and it < 1000:
        x3 = 0.5 * (x2 + x1)
        y3 = f(x3)
        dy = y3 * y3 - y1 * y2
        if dy == 0.0:
            x = x3
            break
        sgn = 0.0 if (y1 - y2) == 0.0 else (1.0 if math.copysign(1.0, y1 - y2) > 0 else -1.0)
        dx = (x3 - x1) * sgn * y3 / math.sqrt(dy)
        x = x3 + dx
        y = f(x)
        same3 = math.copysign(1.0, y) == math.copysign(1.0, y3)
        y2 = y2 if same3 else y3
        x2 = x2 if same3 else x3
        same1 = (math.copysign(1.0, y) == math.copysign(1.0, y1)) or x2 == x3
        y2 = y2 if same1 else y1
        x2 = x2 if same1 else x1
        y1, x1 = y, x
        teps = abs((x - tx) / (tx + x))
        tx = x
        it += 1
    return x


def equilibrium_m(T, Tc, S):
    """m_e(T) = |n| at the root of B_S(3S/(S+1) Tc/T n) - n (brillouin.cu:79-138).

    Returns 1 at T == 0 and 0 above Tc, as the kernel does (brillouin.cu:103-118).
    """
    if T == 0.0:
        return 1.0
    if T > Tc:
        return 0.0
    pre_s = 1.0 if S > INFINITE_SPIN else S / (S + 1.0)
    pre = 3.0 * pre_s * (Tc / T)
    dT = (Tc - T) / Tc
    lo = -0.1 if dT < 0.0004 else 0.01
    hi = 0.5 if dT < 0.0004 else 1.1
    if S > INFINITE_SPIN:
        f = lambda n: float(langevin(pre * n)) - n
    else:
        f = lambda n: float(brillouin(S, pre * n)) - n
    return abs(_ridders(f, lo, hi))


def brillouin_msat0(T, msat0T0_mask, Tc_mask, S_mask, msat0_mul, msat0T0_mul, Tc_mul, S_mul):
    """brillouinKern (brillouin.cu:88-138): msat0 mask = Ms0T0 * m_e(T) / msat0_mul."""
    T = np.asarray(T, dtype=np.float64)
    shape = T.shape
    ms = msat0T0_mul * _mask(msat0T0_mask, shape)
    Tc = Tc_mul * _mask(Tc_mask, shape)
    S = S_mul * _mask(S_mask, shape)
    out = np.zeros(shape)
    cache = {}
    for idx in np.ndindex(shape):
        if ms[idx] == 0.0:
            continue
        if T[idx] == 0.0:
            out[idx] = ms[idx] / msat0_mul
            continue
        if T[idx] > Tc[idx]:
            continue
        key = (float(T[idx]), float(Tc[idx]), float(S[idx]))
        if key not in cache:
            cache[key] = equilibrium_m(*key)
        out[idx] = ms[idx] * cache[key] / msat0_mul
    return out


def kappa(msat0_mask, msat0T0_mask, T, Tc_mask, S_mask, n_mask,
          msat0_mul, msat0T0_mul, Tc_mul, S_mul):
    """Longitudinal susceptibility mask (kappa.cu:15-61).

    k = mul * f/(1-f), f = b W'(m_e b), b = S/(S+1) 3Tc/T, mul = u^2/(S/(S+1) 3Tc n_mask);
    the quantity multiplier Ms0^2 mu0/(n kB) is set by mod_kappa.go:76-89 (see
    ``kappa_multiplier``).
    """
    T = np.asarray(T, dtype=np.float64)
    shape = T.shape
    u = _mask(msat0T0_mask, shape)
    ms = msat0T0_mul * u
    S = S_mul * _mask(S_mask, shape)
    Tc = Tc_mul * _mask(Tc_mask, shape)
    msat0 = msat0_mul * _mask(msat0_mask, shape)
    n = _mask(n_mask, shape)
    out = np.zeros(shape)
    ok = (ms != 0.0) & (T != 0.0)
    for s in np.unique(S[ok]):
        sel = ok & (S == s)
        pre_s = 1.0 if s > INFINITE_SPIN else s / (s + 1.0)
        J0 = 3.0 * Tc[sel]
        mul = u[sel] * u[sel] / (pre_s * J0 * n[sel])
        me = msat0[sel] / ms[sel]
        b = pre_s * J0 / T[sel]
        f = dlangevin(me * b) if s > INFINITE_SPIN else dbrillouin(s, me * b)
        f = b * f
        out[sel] = mul * (f / (1.0 - f))
    return out


def kappa_multiplier(msat0T0_mul, n_mul):
    """mod_kappa.go:76-89: Ms0^2 mu0 / (n kB)."""
    return msat0T0_mul * msat0T0_mul * MU0 / (n_mul * KB)


def thermal_prefactor(T_mul, cellsize, gamma_ll, dt, cutoff_dt, msat0T0_mul):
    """2 kB T_mul / (mu0 V gamma dt_eff Ms0) (mod_brown.go:125-145)."""
    V = cellsize[0] * cellsize[1] * cellsize[2]
    return KB * 2.0 * T_mul / (MU0 * V * gamma_ll * max(cutoff_dt, dt) * msat0T0_mul)


def scale_noise(noise, mu_mask, mu_mul, T_mask, msat0T0_mask, prefactor):
    """temperature_scaleAnisKern (temperature.cu:14-70).

    H_i = sqrt(prefactor * T_mask / Ms0_mask) * sqrt(mu_ii) * N_i(0,1); zero in vacuum.
    """
    shape = noise.shape[1:]
    ms = _mask(msat0T0_mask, shape)
    T = _mask(T_mask, shape)
    mu = np.stack([np.sqrt(mu_mul[c] * _mask(None if mu_mask is None else mu_mask[c], shape))
                   for c in range(3)])
    safe = np.where(ms == 0.0, 1.0, ms)
    pre = np.sqrt(T * prefactor / safe)
    return np.where(ms == 0.0, 0.0, pre * mu * noise)


# ----------------------------------------------------------------------------- heat baths
def qspat(T, k_mask, k_mul, cellsize, pbc):
    """Q = k_mul * sum_d (1/cs_d^2) [k-(T- - T) + k+(T+ - T)] (Qspat.cu:13-103)."""
    k = _mask(k_mask, T.shape)
    inv = [1.0 / (c * c) for c in cellsize]
    return k_mul * laplace_weighted(T, k, inv, pbc)


def qinter(Ti, Tj, G_mask, G_mul):
    """Q_i = G (T_j - T_i) (Qinter.cu:13-28)."""
    G = G_mul if G_mask is None else G_mul * G_mask
    return G * (Tj - Ti)


def div_zero(a, b):
    """a / b, 0 where b == 0; b None means 1 (div.cu:13-23)."""
    if b is None:
        return np.array(a, dtype=np.float64)
    safe = np.where(b == 0.0, 1.0, b)
    return np.where(b == 0.0, 0.0, a / safe)


def dTdt(Q, C_mask, C_mul):
    """dT/dt = (1/C_mul) * Q / C_mask (modules/TM.go:41-59 + div.cu)."""
    pre = 1.0 / C_mul if C_mul != 0.0 else 0.0
    return pre * div_zero(Q, C_mask)


def drude_ce(Te, n_mask, gamma_mask, n_mul, gamma_mul):
    """Ce = (n/Na) gamma Te (mod_ce.go:73-94): value = Te * n_mask * gamma_mask, multiplier
    (n_mul / Na) * gamma_mul.  Returns the physical Ce."""
    v = np.array(Te, dtype=np.float64)
    if n_mask is not None:
        v = v * n_mask
    if gamma_mask is not None:
        v = v * gamma_mask
    return (n_mul / NA) * gamma_mul * v


def pointwise_of(points, arg):
    """Piecewise-linear value of a tabulated function of ``arg``
    (engine/update_pointwiseof.go:31-98).  ``points`` is a list of (x, v0, v1, ...)."""
    if len(points) < 2:
        raise ValueError("Pointwise definition needs at least two points")
    i = 0
    while i < len(points) and points[i][0] < arg:
        i += 1
    if i >= len(points):
        raise ValueError("Out of range of pointwise-defined quantity")
    if arg != points[i][0]:
        if i - 1 < 0:
            return [0.0] * (len(points[0]) - 1)
        x1, x2 = points[i - 1][0], points[i][0]
        v1, v2 = points[i - 1][1:], points[i][1:]
        f = (arg - x1) / (x2 - x1)
        return [a + f * (b - a) for a, b in zip(v1, v2)]
    return list(points[i][1:])


# ----------------------------------------------------------------------------- energies
def energy_term(m, H, msat_mask, msat_mul, weight):
    """weight * Ms0 * sum_i (m . H)_i msat_i (mod_energy.go:101-116, dot.cu:10-25)."""
    w = (m * H).sum(0)
    if msat_mask is not None:
        w = w * msat_mask
    return float(w.sum()) * msat_mul * weight


# ----------------------------------------------------------------------------- remaining MFA / thermal kernels
DEBYE_STEPS = 61          # common_func.h:27 INTMAXSTEPS


def _debye_integrand(x):
    """x^4 e^x / (e^x - 1)^2, 0 for x <= zero (common_func.h:168-173)."""
    if x <= ZERO:
        return 0.0
    ex = math.exp(x)
    return x ** 4 * ex / ((ex - 1.0) * (ex - 1.0))


def debye_cp(T, Td_mask, n_mask, Td_mul):
    """Debye phonon heat capacity per cell (cpKern, Cp.cu:13-88): n (T/Td)^3 times the
    integral of x^4 e^x/(e^x-1)^2 over [0, Td/T] by the composite trapezoid rule on 61
    intervals; the T/Td < 0.01 limit n (12/5)(1/9) pi^4 (T/Td)^3; 0 where Td = 0."""
    T = np.asarray(T, dtype=np.float64)
    out = np.zeros_like(T)
    Td = Td_mul * _mask(Td_mask, T.shape)
    n = _mask(n_mask, T.shape)
    for idx in np.ndindex(T.shape):
        td, t = Td[idx], T[idx]
        if td == 0.0:
            continue
        xx, ixx = td / t, t / td
        if ixx < 0.01:
            out[idx] = n[idx] * (12.0 / 5.0) * (1.0 / 9.0) * math.pi ** 4 * ixx ** 3
            continue
        h = xx / DEBYE_STEPS
        inner = sum(_debye_integrand(j * h) for j in range(1, DEBYE_STEPS))
        val = (_debye_integrand(0.0) + _debye_integrand(DEBYE_STEPS * h) + 2.0 * inner) * 0.5 * h
        out[idx] = n[idx] * val / xx ** 3
    return out


def spin_temperature(msat_mask, msat0T0_mask, Tc_mask, S_mask, msat_mul, msat0T0_mul, Tc_mul, S_mul, shape):
    """Temperature whose mean-field equilibrium gives m = msat/Msat0T0 (tsKern, Ts.cu:84-125):
    root of B_S(S^2 J0 m / T) - m on [0, Tc] by Ridders, J0 = 3 Tc/(S(S+1)); 0 where
    Msat0T0 = 0 or msat = Msat0T0, Tc where msat = 0."""
    out = np.zeros(shape)
    ms = msat_mul * _mask(msat_mask, shape)
    ms0 = msat0T0_mul * _mask(msat0T0_mask, shape)
    Tc = Tc_mul * _mask(Tc_mask, shape)
    S = S_mul * _mask(S_mask, shape)
    for idx in np.ndindex(shape):
        if ms0[idx] == 0.0 or ms[idx] == ms0[idx]:
            continue
        if ms[idx] == 0.0:
            out[idx] = Tc[idx]
            continue
        s, tc = S[idx], Tc[idx]
        m = ms[idx] / ms0[idx]
        pre = s * s * (3.0 * tc / (s * (s + 1.0))) * m
        out[idx] = _ridders(lambda t: float(brillouin(s, 1.0e38 if t == 0.0 else pre / t)) - m, 0.0, tc)
    return out


def weighted_avg(a, b, w0_mask, w1_mask, R_mask, w0_mul, w1_mul, R_mul):
    """(w0 a + w1 b + 2R sqrt(w0 a w1 b)) / (w0 + w1 + 2R sqrt(w0 w1)), 0 where the
    denominator vanishes (wavgKern, wavg.cu:13-30; common_func.h:162-166)."""
    shape = np.shape(a)
    w0 = w0_mul * _mask(w0_mask, shape)
    w1 = w1_mul * _mask(w1_mask, shape)
    R = R_mul * _mask(R_mask, shape)
    den = w0 + w1 + 2.0 * R * np.sqrt(w0 * w1)
    num = w0 * a + w1 * b + 2.0 * R * np.sqrt(w0 * a * w1 * b)
    return np.where(den == 0.0, 0.0, num / np.where(den == 0.0, 1.0, den))


def energy_flow(m, R, Tc_mask, S_mask, n_mask, S_mul):
    """Tc S^2 n / (S(S+1)) (m . R) with Tc and n from their masks alone (energyFlowKern,
    energy_flow.cu:15-44); 0 where n, S or Tc is 0."""
    shape = m.shape[1:]
    S = S_mul * _mask(S_mask, shape)
    Tc = _mask(Tc_mask, shape)
    n = _mask(n_mask, shape)
    ok = (n != 0.0) & (S != 0.0) & (Tc != 0.0)
    Ss = np.where(ok, S, 1.0)
    mult = Tc * Ss * Ss * n / (Ss * (Ss + 1.0))
    return np.where(ok, mult * (m * R).sum(0), 0.0)


def llbar_nonlocal00nc(h, msat0T0_mask, lam_masks, lam_mul, cellsize, pbc):
    """Nonlocal (exchange-like) damping torque (llbarNonlocal00ncKern,
    llbar-nonlocal00nc.cu:11-205): t_c = -sum_d lam_c/cs_d^2 ((l1 H1 + l2 H2) - H0 (l1 + l2))
    with l1, l2 the harmonic means of the lambda_e mask of the cell and each neighbour
    (per component), clamp/wrap boundaries, 0 where Msat0T0 = 0.  The reference computes the
    a1 + 1 neighbour's index with N1 in place of N2; this restatement uses the grid's index
    (the two agree when N1 == N2)."""
    shape = h.shape[1:]
    out = np.zeros_like(h)
    for c in range(3):
        lm = _mask(lam_masks[c] if lam_masks is not None else None, shape)
        acc = np.zeros(shape)
        for d in range(3):
            lo = np.take(lm, _neighbour_index(shape[d], pbc[d], -1), axis=d)
            hi = np.take(lm, _neighbour_index(shape[d], pbc[d], +1), axis=d)
            Hlo = np.take(h[c], _neighbour_index(shape[d], pbc[d], -1), axis=d)
            Hhi = np.take(h[c], _neighbour_index(shape[d], pbc[d], +1), axis=d)
            l1, l2 = avg_geom_zero(lm, lo), avg_geom_zero(lm, hi)
            acc += lam_mul[c] / (cellsize[d] ** 2) * ((l1 * Hlo + l2 * Hhi) - h[c] * (l1 + l2))
        out[c] = -acc
    if msat0T0_mask is not None:
        out = np.where(np.asarray(msat0T0_mask)[None] == 0.0, 0.0, out)
    return out
