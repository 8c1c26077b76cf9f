"""Script-level mirror of hotspin's Python client API, on the B200 simulation handle.

hotspin scripts (``python/hotspin.py``, generated from ``engine/api.go``) build a module graph
with ``load(...)`` and set quantities with ``setv``/``setmask``/``setarray``; the Go engine
then steps it.  This module accepts the same calls for the modules of the solver hot path
and runs them on ``hsb_sim`` (one fused, device-resident step).  User-facing order is the
reference's: ``setgridsize(x, y, z)`` and vectors ``[x, y, z]``; arrays are
``array[c][i][j][k]`` with i = x (``python/hotspin.py`` ``makearray``).  Internally
everything is converted to program order (z, y, x) exactly as ``engine/api.go:41-62`` and
``common/index.go:68-113`` do.

Supported modules: exchange6, demag, zeeman, anisotropy/uniaxial, llbar, llbar/torque,
llbar/damping/nonconservative/00/local, llbar/damping/nonconservative/02/local (setv('μ∥',
...)), llbar/damping/conservative/02/local (setv('μ⊥', ...)),
llbar/damping/nonconservative/00/nonlocal (setv('αₑ', ...)), normalizer, mfa/longfield, mfa/msat0,
temperature/brown, temperature/ETM, temperature/PTM, temperature/E-P, temperature/Drude,
temperature/ETM/diffusion, solver/euler, solver/heun, solver/rk12 (errors per step set with
setv('m_maxerror' / 'Te_maxerror' / 'Tp_maxerror', ...)), solver/am12 ('<q>_maxabserror',
'<q>_maxrelerror'), solver/bdf-euler ('m_maxitererror', 'm_maxiterations'), solver/rk4,
solver/rk45, micromag/energy.  Anything else raises (no silent fallback).
"""
import math

import numpy as np

from .sim import Simulation

MU0 = 4.0 * math.pi * 1e-7
MUB = 9.27400968202020202e-24

SUPPORTED = {
    "exchange6", "demag", "zeeman", "anisotropy/uniaxial", "llbar", "llbar/torque",
    "llbar/damping/nonconservative/00/local", "llbar/damping/nonconservative/02/local",
    "llbar/damping/conservative/02/local", "llbar/damping/nonconservative/00/nonlocal", "normalizer",
    "mfa/longfield", "mfa/msat0",
    "temperature/brown", "temperature/ETM", "temperature/PTM", "temperature/E-P",
    "temperature/Drude", "temperature/ETM/diffusion", "solver/euler", "solver/heun",
    "solver/rk12", "solver/am12", "solver/bdf-euler", "solver/rk4", "solver/rk45", "micromag/energy",
}


def _swap3(v):
    """user (x, y, z) -> program (z, y, x)"""
    return (float(v[2]), float(v[1]), float(v[0]))


def _to_program_scalar(a):
    """user array [i][j][k] (x, y, z) -> program [z][y][x]"""
    return np.ascontiguousarray(np.transpose(np.asarray(a, dtype=np.float64), (2, 1, 0)))


def _to_program_vector(a):
    a = np.asarray(a, dtype=np.float64)
    return np.stack([_to_program_scalar(a[2]), _to_program_scalar(a[1]), _to_program_scalar(a[0])])


def _to_user_vector(p):
    t = lambda x: np.ascontiguousarray(np.transpose(x, (2, 1, 0)))
    return np.stack([t(p[2]), t(p[1]), t(p[0])])


class Engine:
    """One hotspin-like engine; the module-level functions below drive a default one."""

    def __init__(self):
        self.size = None          # program order
        self.cellsize = None
        self.pbc = (0, 0, 0)
        self.modules = set()
        self.v = {}
        self.masks = {}
        self.arrays = {}
        self.t = 0.0
        self.sim = None

    # ---------------------------------------------------------------- geometry
    def setgridsize(self, x, y, z):
        self.size = (int(z), int(y), int(x))
        self._reset()

    def setcellsize(self, x, y, z):
        self.cellsize = (float(z), float(y), float(x))
        self._reset()

    def setperiodic(self, x, y, z):
        self.pbc = (int(z), int(y), int(x))
        self._reset()

    # ---------------------------------------------------------------- modules / values
    def load(self, name):
        if name not in SUPPORTED:
            raise ValueError("module %r is not part of the B200 hot path" % name)
        self.modules.add(name)
        self._reset()

    def setv(self, name, value):
        if isinstance(value, (list, tuple)) and len(value) == 3:
            value = _swap3(value)
        self.v[name] = value
        if name in ("dt", "t"):
            if self.sim is not None:
                self.sim.set_time(self.v.get("t", self.t) if name == "t" else self._status()["t"],
                                  self.v["dt"] if name == "dt" else 0.0)
            if name == "t":
                self.t = float(value)
            return
        self._reset()

    def getv(self, name):
        if name == "t":
            return self._status()["t"] if self.sim else self.t
        if name == "dt":
            return self._status()["dt"] if self.sim else self.v.get("dt")
        if name == "E":
            return self._sim().energy()
        if name == "<m>":
            return list(_swap3(self._sim().average_m()))
        v = self.v[name]
        return list(_swap3(v)) if isinstance(v, tuple) and len(v) == 3 else v

    def setmask(self, name, arr):
        key = name.lower()
        if key not in ("msat0t0", "lex", "msat0"):
            raise ValueError("mask %r is not supported on the B200 path" % name)
        if key == "msat0":
            return                      # msat0 is derived from msat0T0 and m_e(T) here
        self.masks[key] = _to_program_scalar(np.asarray(arr)[0] if np.asarray(arr).ndim == 4 else arr)
        self._reset()

    def setarray(self, name, arr):
        a = np.asarray(arr, dtype=np.float64)
        if name == "m":
            self.arrays["m"] = _to_program_vector(a)
        elif name in ("Te", "Tp"):
            s = a[0] if a.ndim == 4 else a
            if s.size == 1:
                s = np.full(tuple(reversed(self.size)), float(s.ravel()[0]))
            self.arrays["Te" if name == "Te" else "Tl"] = _to_program_scalar(s)
        else:
            raise ValueError("array %r is not supported on the B200 path" % name)
        if self.sim is not None:
            self.sim.set("m" if name == "m" else ("Te" if name == "Te" else "Tl"),
                         self.arrays["m" if name == "m" else ("Te" if name == "Te" else "Tl")])

    def getarray(self, name):
        sim = self._sim()
        if name == "m":
            return _to_user_vector(sim.get("m"))
        if name == "B":
            return _to_user_vector(sim.get("H_demag") * MU0)
        if name in ("Te", "Tp"):
            return np.ascontiguousarray(np.transpose(sim.get("Te" if name == "Te" else "Tl"), (2, 1, 0)))[None]
        raise ValueError("array %r is not available on the B200 path" % name)

    # ---------------------------------------------------------------- time stepping
    def step(self, n=1):
        self._sim().step(n)

    def run(self, duration):
        self.run_until(self.getv("t") + duration)

    def run_until(self, t):
        self._sim().run_until(t)

    # ---------------------------------------------------------------- internals
    def _reset(self):
        if self.sim is not None:
            self.sim.close()
            self.sim = None

    def _status(self):
        return self.sim.status()

    def _desc(self):
        g = lambda k, d=0.0: self.v.get(k, d)
        mods = self.modules
        msat = g("Msat0T0", g("msat0T0", 0.0))
        solver = "rk4"
        for s in ("euler", "heun", "rk12", "am12", "bdf-euler", "rk4", "rk45"):
            if "solver/" + s in mods:
                solver = "dp45" if s == "rk45" else s
        # quantity names are matched without case, as the reference's engine does
        lv = {k.lower(): v for k, v in self.v.items()}
        per_eq = lambda suffix: (float(lv.get("m_" + suffix, 0.0)), float(lv.get("te_" + suffix, 0.0)),
                                 float(lv.get("tp_" + suffix, lv.get("tl_" + suffix, 0.0))))
        if solver == "am12":
            maxerr, maxrelerr = per_eq("maxabserror"), per_eq("maxrelerror")
        elif solver == "bdf-euler":
            maxerr, maxrelerr = per_eq("maxitererror"), (0.0, 0.0, 0.0)
        else:
            maxerr, maxrelerr = per_eq("maxerror"), (0.0, 0.0, 0.0)
        max_iter = int(lv.get("m_maxiterations", 0))
        d = dict(size=self.size, cellsize=self.cellsize, pbc=self.pbc, msat0T0=msat,
                 lex=g("lex") if "exchange6" in mods else 0.0,
                 gamma_ll=g("γ_LL", g("γ_ll", 2.211e5)),
                 alpha=g("α", (0.0, 0.0, 0.0)) if "llbar/damping/nonconservative/00/local" in mods else (0, 0, 0),
                 ku=g("Ku") if "anisotropy/uniaxial" in mods else 0.0, anis_u=g("anisU", (0.0, 0.0, 1.0)),
                 b_ext=g("B_ext", (0.0, 0.0, 0.0)) if "zeeman" in mods else (0.0, 0.0, 0.0),
                 demag="demag" in mods, normalize="normalizer" in mods, llb="mfa/longfield" in mods,
                 tc=g("Tc"), spin_j=g("J", 0.5), n_spins=g("n"), temperature=g("Temp", 0.0),
                 thermal="temperature/brown" in mods, seed=int(g("Therm_seed", 0)), cutoff_dt=g("cutoff_dt"),
                 ttm="temperature/ETM" in mods, solver=solver, dt=g("dt", 1e-15), rtol=g("m_maxrelerror", 1e-5),
                 mindt=g("mindt", 1e-22), maxdt=g("maxdt", 1e-12), maxerr=maxerr, maxrelerr=maxrelerr,
                 max_iter=max_iter,
                 mu_par=g("μ∥", (0.0, 0.0, 0.0)) if "llbar/damping/nonconservative/02/local" in mods else (0, 0, 0),
                 mu_perp=g("μ⊥", (0.0, 0.0, 0.0)) if "llbar/damping/conservative/02/local" in mods else (0, 0, 0),
                 alpha_e=g("αₑ", (0.0, 0.0, 0.0)) if "llbar/damping/nonconservative/00/nonlocal" in mods else (0, 0, 0))
        if d["ttm"]:
            d.update(gamma_e=g("γ") * g("n") / 6.02214129272727272e23 if "temperature/Drude" in mods else 0.0,
                     c_l=g("Cp"), g_ep=g("Ge-p"), k_e=g("Ke") if "temperature/ETM/diffusion" in mods else 0.0)
        if msat == 0.0 or self.size is None or self.cellsize is None:
            raise ValueError("setgridsize, setcellsize and setv('Msat0T0', ...) are required")
        return d

    def _sim(self):
        if self.sim is None:
            self.sim = Simulation(**self._desc())
            if "msat0t0" in self.masks:
                self.sim.set("msat_mask", self.masks["msat0t0"])
            if "lex" in self.masks:
                self.sim.set("lex_mask", self.masks["lex"])
            for k, v in self.arrays.items():
                self.sim.set(k, v)
            if self.t:
                self.sim.set_time(self.t, 0.0)
        return self.sim


_default = Engine()


def _bind(name):
    def f(*a, **k):
        return getattr(_default, name)(*a, **k)
    f.__name__ = name
    f.__doc__ = getattr(Engine, name).__doc__
    return f


for _n in ("setgridsize", "setcellsize", "setperiodic", "load", "setv", "getv", "setmask", "setarray",
           "getarray", "step", "run", "run_until"):
    globals()[_n] = _bind(_n)


def makearray(ncomp, nx, ny, nz):
    """python/hotspin.py makearray: nested list [c][i][j][k]."""
    return np.zeros((ncomp, nx, ny, nz)).tolist()


def new_engine():
    """A fresh engine (the module-level functions use a shared default one)."""
    return Engine()
