"""FP64 right-hand side of the hotspin LLBar / LLB / two-temperature problem (test infrastructure).

Assembles the terms the way hotspin's module graph does for the scripts the configurations
describe (tests/stdproblem4-llbr-modular.py, examples/laser-demag.py):

* H_eff = H_ex + H_anis + B_ext/mu0 + B_demag/mu0 + H_lf + H_therm
  (SumUpdater over the loaded terms: engine/update_sum.go:29-76, modules/hfield.go:19-28,
  mod_zeeman.go:23-31, mod_demag.go:56-62);
* dm/dt = llbar_torque + llbar_local00nc = gamma_LL (m x H) + gamma_LL diag(lambda) H
  (the reference's ``cross(H, M)`` helper evaluates m x H, common_func.h:52-55)
  (modules/mod_llbar.go:29-38, llbar-torque.cu:11-45, llbar-local00nc.cu:11-63);
* with the ``normalizer`` module (LLG mode) m is renormalised whenever it is updated, i.e.
  before every right-hand-side evaluation (mod_normalize.go:45-55, engine/quant.go:417-445);
* two-temperature model: C_e dTe/dt = k_e lap(Te) + G (Tl - Te) + Q_laser,
  C_l dTl/dt = k_l lap(Tl) + G (Te - Tl) (modules/TM.go:15-59, Qspat.cu, Qinter.cu,
  mod_ce.go:73-94 with C_e = gamma_e Te).

``Spec`` fields are in program order (slow -> fast = user z, y, x).
"""
import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import fields as F
from .demag import DemagPlan
from .philox import thermal_normals


@dataclass
class Spec:
    size: tuple                      # (N0, N1, N2) program order
    cellsize: tuple                  # metres, program order
    pbc: tuple = (0, 0, 0)
    msat0T0: float = 8.0e5           # A/m
    lex: float = 0.0                 # exchange length multiplier (m)
    gamma_ll: float = F.GAMMA0
    alpha: tuple = (0.0, 0.0, 0.0)   # lambda diagonal (program components)
    ku: float = 0.0
    anis_u: tuple = (0.0, 0.0, 1.0)  # program components
    b_ext: tuple = (0.0, 0.0, 0.0)   # tesla, program components
    demag: bool = False
    normalize: bool = False
    llb: bool = False
    tc: float = 0.0
    spin_j: float = 0.5
    n_spins: float = 0.0
    temperature: float = 0.0         # uniform bath temperature (used when ttm is False)
    thermal: bool = False
    seed: int = 0
    cutoff_dt: float = 0.0
    ttm: bool = False
    gamma_e: float = 0.0             # J/(m^3 K^2): Ce = gamma_e Te
    c_l: float = 0.0                 # J/(m^3 K)
    g_ep: float = 0.0                # W/(m^3 K)
    k_e: float = 0.0                 # W/(m K)
    k_l: float = 0.0
    laser_p0: float = 0.0            # W/m^3 peak
    laser_t0: float = 0.0            # s, pulse centre
    laser_fwhm: float = 1.0e-13      # s
    laser_sigma: float = 0.0         # m, lateral Gaussian spot (0 = uniform)
    laser_table: object = None       # (t, factor) pairs: pointwise time profile instead of the Gaussian
    bext_table: object = None        # (t, Bx, By, Bz) rows (tesla): pointwise applied field instead of b_ext
    msat_mask: Optional[np.ndarray] = None
    lex_mask: Optional[np.ndarray] = None
    mu_par: tuple = (0.0, 0.0, 0.0)  # llbar/damping/nonconservative/02/local (program components)
    mu_perp: tuple = (0.0, 0.0, 0.0)  # llbar/damping/conservative/02/local
    alpha_e: tuple = (0.0, 0.0, 0.0)  # llbar/damping/nonconservative/00/nonlocal


def laser_profile(spec):
    """Lateral spot shape (N0, N1, N2): Gaussian in the program Y/Z (user y/x) plane about
    the grid centre, uniform through the thickness; 1 everywhere when sigma == 0."""
    n0, n1, n2 = spec.size
    if spec.laser_sigma <= 0.0:
        return np.ones(spec.size)
    y = (np.arange(n1) + 0.5 - 0.5 * n1) * spec.cellsize[1]
    x = (np.arange(n2) + 0.5 - 0.5 * n2) * spec.cellsize[2]
    r2 = y[:, None] ** 2 + x[None, :] ** 2
    g = np.exp(-r2 / (2.0 * spec.laser_sigma ** 2))
    return np.broadcast_to(g[None], spec.size).copy()


def bext_at(spec, t):
    """Applied field (tesla, program components) at time t: b_ext, or the piecewise-linear
    interpolation of the (t, B) table (engine/update_pointwiseof.go:31-98), zero outside it."""
    if spec.bext_table is None or t is None:
        return np.asarray(spec.b_ext, dtype=np.float64)
    tab = np.asarray(spec.bext_table, dtype=np.float64).reshape(-1, 4)
    if t < tab[0, 0] or t > tab[-1, 0]:
        return np.zeros(3)
    i = int(np.searchsorted(tab[:, 0], t, side="right")) - 1
    i = min(max(i, 0), len(tab) - 2)
    f = (t - tab[i, 0]) / (tab[i + 1, 0] - tab[i, 0])
    return tab[i, 1:] + f * (tab[i + 1, 1:] - tab[i, 1:])


def laser_time(spec, t):
    """Time factor of the absorbed power: a Gaussian with the given FWHM, peak 1 at t0; or,
    with a (t, factor) table, its piecewise-linear interpolation as a hotspin pointwise
    quantity (engine/update_pointwiseof.go:31-98), zero outside the table's time range."""
    if spec.laser_table is not None:
        tab = np.asarray(spec.laser_table, dtype=np.float64).reshape(-1, 2)
        if t < tab[0, 0] or t > tab[-1, 0]:
            return 0.0
        i = int(np.searchsorted(tab[:, 0], t, side="right")) - 1
        i = min(max(i, 0), len(tab) - 2)
        (t1, v1), (t2, v2) = tab[i], tab[i + 1]
        return float(v1 + (t - t1) / (t2 - t1) * (v2 - v1))
    s = (t - spec.laser_t0) / spec.laser_fwhm
    return math.exp(-4.0 * math.log(2.0) * s * s)


class Model:
    """RHS evaluator.  State y: dict with 'm' (3, N0, N1, N2) and, with ttm, 'Te', 'Tl'."""

    def __init__(self, spec: Spec):
        self.s = spec
        self.plan = DemagPlan(spec.size, spec.cellsize, spec.pbc) if spec.demag else None
        self.spot = laser_profile(spec) if spec.ttm else None
        self.ncell = int(np.prod(spec.size))
        self.noise = None          # H_therm held for the current step
        self.noise_key = None

    # -- thermal field ------------------------------------------------------------
    def set_thermal(self, step, dt, T):
        """Generate H_therm for one step (mod_brown.go:103-149): fresh normals per step,
        scaled with the step's dt; mu = lambda (isotropic thermal tensor)."""
        s = self.s
        if not s.thermal:
            self.noise = None
            return
        if self.noise_key != step:
            self._normals = thermal_normals(self.ncell, step, s.seed).reshape((3,) + tuple(s.size))
            self.noise_key = step
        pre = F.thermal_prefactor(1.0, s.cellsize, s.gamma_ll, dt, s.cutoff_dt, s.msat0T0)
        Tm = np.broadcast_to(np.asarray(T, dtype=np.float64), s.size)
        self.noise = F.scale_noise(self._normals, None, s.alpha, Tm, s.msat_mask, pre)

    def spin_temperature(self, y):
        return y["Te"] if self.s.ttm else np.full(self.s.size, self.s.temperature)

    # -- fields -------------------------------------------------------------------
    def heff_terms(self, y):
        s = self.s
        m = y["m"]
        terms = {}
        if s.lex != 0.0:
            terms["H_ex"] = F.exchange6(m, s.lex_mask, s.msat0T0, s.lex, s.cellsize, s.pbc)
        if s.ku != 0.0:
            terms["H_anis"] = F.uniaxial_anisotropy(m, None, s.msat_mask, s.ku, s.msat0T0,
                                                    None, s.anis_u)
        if self.plan is not None:
            terms["B"] = self.plan.field(m, s.msat_mask, s.msat0T0)
        if s.llb:
            T = self.spin_temperature(y)
            terms["H_lf"] = F.long_field(m, s.msat_mask, None, None, None, T,
                                         s.msat0T0, s.spin_j, s.n_spins, s.tc, 1.0)
        return terms

    def heff(self, y, time=None):
        s = self.s
        t = self.heff_terms(y)
        H = np.zeros_like(y["m"])
        for name, v in t.items():
            H += v / F.MU0 if name == "B" else v
        b = bext_at(s, time)
        for c in range(3):
            H[c] += b[c] / F.MU0
        if self.noise is not None:
            H += self.noise
        return H

    def rhs(self, t, y):
        s = self.s
        m = F.normalize(y["m"]) if s.normalize else y["m"]
        yy = dict(y)
        yy["m"] = m
        H = self.heff(yy, t)
        dm = F.llbar_torque(m, H, s.msat_mask, s.gamma_ll)
        dm = dm + F.llbar_local00nc(H, s.msat_mask, None, s.alpha, s.gamma_ll)
        if any(v != 0.0 for v in s.mu_par):
            dm = dm + F.llbar_local02nc(m, H, s.msat_mask, None, s.mu_par, s.gamma_ll)
        if any(v != 0.0 for v in s.mu_perp):
            dm = dm + F.llbar_local02c(m, H, s.msat_mask, None, s.mu_perp, s.gamma_ll)
        if any(v != 0.0 for v in s.alpha_e):
            dm = dm + s.gamma_ll * F.llbar_nonlocal00nc(H, s.msat_mask, None, s.alpha_e, s.cellsize, s.pbc)
        out = {"m": dm}
        if s.ttm:
            Te, Tl = y["Te"], y["Tl"]
            Qe = F.qspat(Te, None, s.k_e, s.cellsize, s.pbc) + F.qinter(Te, Tl, None, s.g_ep)
            Qe = Qe + s.laser_p0 * laser_time(s, t) * self.spot
            Ql = F.qinter(Tl, Te, None, s.g_ep)
            if s.k_l != 0.0:
                Ql = Ql + F.qspat(Tl, None, s.k_l, s.cellsize, s.pbc)
            Ce = s.gamma_e * Te
            out["Te"] = F.div_zero(Qe, Ce)
            out["Tl"] = Ql / s.c_l if s.c_l != 0.0 else np.zeros_like(Tl)
        return out

    # -- energy -------------------------------------------------------------------
    def energy(self, y, time=None):
        """Total micromagnetic energy as mod_energy.go:20-66 sums it (J), with the applied
        field at `time` when it is given pointwise."""
        s = self.s
        m = F.normalize(y["m"]) if s.normalize else y["m"]
        yy = dict(y)
        yy["m"] = m
        V = float(np.prod(s.cellsize))
        t = self.heff_terms(yy)
        E = 0.0
        b_now = bext_at(s, time)
        bext = np.stack([np.full(s.size, b) for b in b_now])
        if any(b != 0.0 for b in b_now):
            E += F.energy_term(m, bext, s.msat_mask, s.msat0T0, -V)
        if "H_ex" in t:
            E += F.energy_term(m, t["H_ex"], s.msat_mask, s.msat0T0, -0.5 * V * F.MU0)
        if "B" in t:
            E += F.energy_term(m, t["B"], s.msat_mask, s.msat0T0, -0.5 * V)
        if "H_anis" in t:
            E += F.energy_term(m, t["H_anis"], s.msat_mask, s.msat0T0, -0.5 * V * F.MU0)
        if "H_lf" in t:
            E += F.energy_term(m, t["H_lf"], s.msat_mask, s.msat0T0, -V * F.MU0)
        return E
