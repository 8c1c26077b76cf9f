"""FP64 time integrators (test infrastructure).

* ``euler``, ``heun``, ``rk12`` restate the reference solvers (engine/solve_euler.go:22-50,
  solve_heun.go:27-79, solve_rk12.go:91-214), including the in-place renormalisation that
  the ``normalizer`` module applies each time m is updated (engine/quant.go:417-445).
* ``rk4`` and ``dp45`` are integrators the reference does not have; they use the same
  right-hand side and the same renormalisation rule: every stage point and every accepted
  state is renormalised before it is used (LLG mode only).

DP45 (Dormand-Prince 5(4), first-same-as-last) error norm, per equation:
  m:  max_i |e_i| / rtol                       (m is reduced by Ms0, |m| <= 1)
  T:  max_i |e_i| / (rtol * max(|T0_i|, |T1_i|))
err = max over equations; accept when err <= 1;
dt_new = dt * clamp(0.9 err^-1/5, 0.2, 5) after an accepted step, clamp(., 0.2, 1) after a
rejected one, then clamped to [mindt, maxdt]; a step at mindt is always accepted.
"""
import math

import numpy as np

from . import fields as F

DP_C = [0.0, 1 / 5, 3 / 10, 4 / 5, 8 / 9, 1.0, 1.0]
DP_A = [
    [],
    [1 / 5],
    [3 / 40, 9 / 40],
    [44 / 45, -56 / 15, 32 / 9],
    [19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729],
    [9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656],
    [35 / 384, 0.0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84],
]
DP_B = DP_A[6] + [0.0]
DP_BS = [5179 / 57600, 0.0, 7571 / 16695, 393 / 640, -92097 / 339200, 187 / 2100, 1 / 40]
DP_E = [b - bs for b, bs in zip(DP_B, DP_BS)]


def _comb(y0, ks, coefs, h):
    out = {}
    for key in y0:
        acc = np.zeros_like(y0[key])
        for c, k in zip(coefs, ks):
            if c != 0.0:
                acc = acc + c * k[key]
        out[key] = y0[key] + h * acc
    return out


def rk12_rule(dt, errs, limits, mindt, maxdt):
    """The step-size rule of solve_rk12.go:148-199 for one attempt: errs[q] = dt max|k1 - k0|
    of equation q, limits[q] its maxError, visited in order with the running bad-step flag.
    Returns (accept, bad, dt_new, max errs[q] / limits[q])."""
    bad = False
    fmin = 2.0
    emax = 0.0
    for err, lim in zip(errs, limits):
        if err > lim:
            bad = True
        r = lim / err if err > 0 else math.inf
        fac = r ** (1.0 / 3.0) if bad else math.sqrt(r)
        fac = min(max(fac * 0.8, 0.1), 1.5)
        fmin = min(fmin, fac)
        emax = max(emax, err / lim)
    newdt = min(max(dt * fmin, mindt), maxdt)
    return (not bad) or newdt == mindt, bad, newdt, emax


def _div(a, b):
    """a / b with IEEE results for b == 0 (inf, or nan for 0 / 0), as Go's float64 division."""
    if b == 0.0:
        return math.nan if a == 0.0 or a != a else math.copysign(math.inf, a)
    return a / b


def am_error(a, b, scale, abs_err, rel_err):
    """The error norm of solver/am12 (solve_am01.go:120-131, 247-256): per component p,
    MaxDiff(a_p, b_p) / (maxAbsError + MaxAbs(scale_p) maxRelError), root mean square over
    the components.  The iterators compare the previous iterate with the new one (scale: the
    new one); the step error compares the corrector with the predictor (scale: predictor)."""
    comps = a.shape[0] if a.ndim == 4 else 1
    av, bv, sv = a.reshape(comps, -1), b.reshape(comps, -1), scale.reshape(comps, -1)
    t = 0.0
    for c in range(comps):
        d = float(np.abs(av[c] - bv[c]).max())
        mx = float(np.abs(sv[c]).max())
        t += _div(d, abs_err + mx * rel_err) ** 2
    return math.sqrt(t) / math.sqrt(comps)


def am_iter_rule(er, terrs):
    """One fixed-point iteration's bookkeeping (solve_am01.go:116-150): alpha_i = tErr_i / er_i
    against the error list of the previous iteration, er_i = tErr_i, then the list is sorted in
    place (so the next iteration pairs tErr_i with the i-th smallest error); returns
    (new er, per-equation alphas, err = max, alpha = max)."""
    alp = [_div(t, e) for t, e in zip(terrs, er)]
    er = sorted(terrs)
    return er, alp, er[-1], max(alp)


class Integrator:
    """Drives a ``Model``.  ``y`` is a dict of arrays; ``t``, ``dt``, ``step`` as in the
    reference engine (engine/engine.go:473-508)."""

    def __init__(self, model, y, method, dt, rtol=1e-5, mindt=1e-20, maxdt=1e-10,
                 maxerr=1e-4, t=0.0, maxabserr=None, maxrelerr=None, max_iter=3, max_iter_err=1e-5):
        self.model = model
        self.norm = model.s.normalize
        self.y = {k: np.array(v, dtype=np.float64) for k, v in y.items()}
        if self.norm:
            self.y["m"] = F.normalize(self.y["m"])
        self.method = method
        self.t = t
        self.dt = dt
        self.step_count = 0
        self.rtol = rtol
        self.mindt = mindt
        self.maxdt = maxdt
        self.maxerr = maxerr
        # am12: per-equation absolute / relative error limits (the reference's defaults)
        self.maxabserr = {k: 1e-4 for k in self.y} if maxabserr is None else dict(maxabserr)
        self.maxrelerr = {k: 1e-3 for k in self.y} if maxrelerr is None else dict(maxrelerr)
        # bdf-euler: iterations and iterator error per equation (defaults 3, 1e-5)
        self.max_iter = max_iter
        self.max_iter_err = max_iter_err
        self.iterations = 0
        self.bad_steps = 0
        self.k_fsal = None
        self.last_err = 0.0

    def _fix(self, y):
        if self.norm:
            y = dict(y)
            y["m"] = F.normalize(y["m"])
        return y

    def _thermal(self, dt):
        T = self.model.spin_temperature(self.y)
        self.model.set_thermal(self.step_count, dt, T)

    def step(self):
        getattr(self, "_" + self.method)()

    def run_steps(self, n):
        for _ in range(n):
            self.step()

    def run_until(self, t_end):
        """Step until t_end; adaptive steps are clamped to land on it (as the device does)."""
        while t_end - self.t > 1e-6 * self.dt:
            if self.method in ("dp45", "rk12", "am12"):
                self.dt = min(self.dt, t_end - self.t)
            self.step()

    # -- reference solvers --------------------------------------------------------
    def _euler(self):
        f = self.model.rhs
        self._thermal(self.dt)
        k = f(self.t, self.y)
        self.y = self._fix(_comb(self.y, [k], [1.0], self.dt))
        self.t += self.dt
        self.step_count += 1

    def _heun(self):
        f, h = self.model.rhs, self.dt
        self._thermal(h)
        k0 = f(self.t, self.y)
        y1 = self._fix(_comb(self.y, [k0], [1.0], h))
        self.t += h
        k1 = f(self.t, y1)
        self.y = self._fix(_comb(y1, [k1, k0], [0.5, -0.5], h))
        self.step_count += 1

    def _rk12_limits(self):
        """Per-equation error limits: a float applies to m (and to every equation when it is
        the only limit given); a dict maps equation names (m, Te, Tl) to limits, a missing or
        non-positive temperature entry leaving that equation uncontrolled."""
        me = self.maxerr
        if isinstance(me, dict):
            return [(k, me.get(k, 0.0) if me.get(k, 0.0) > 0 else math.inf) for k in ("m", "Te", "Tl") if k in self.y]
        return [(k, me) for k in ("m", "Te", "Tl") if k in self.y]

    def _rk12(self):
        """solve_rk12.go:91-214.  k0 = f(y0) once per step (the reference restores it on a
        retry; recomputing gives the same values), Euler predictor y1 (renormalised),
        Heun corrector y1 + dt/2 (k1 - k0); per equation err = dt max|k1 - k0|, visited in
        the order m, Te, Tl with the reference's running bad-step flag (a bad equation and
        every later one take the cube-root factor, the others the square root), factor x 0.8
        clamped to [0.1, 1.5], the smallest over the equations; dt_new clamped to
        [mindt, maxdt]; the attempt is kept when no equation was bad or dt_new == mindt;
        the 12th bad attempt of a step raises, as the reference panics.  The thermal field
        is drawn for each attempt with the attempt's dt (as the device does)."""
        f = self.model.rhs
        t0 = self.t
        y0 = self.y
        limits = self._rk12_limits()
        tr = 0
        while True:
            dt = self.dt
            self._thermal(dt)
            k0 = f(t0, y0)
            y1 = self._fix(_comb(y0, [k0], [1.0], dt))
            k1 = f(t0 + dt, y1)
            ynew = self._fix(_comb(y1, [k1, k0], [0.5, -0.5], dt))
            errs = [float(np.abs(k1[key] - k0[key]).max()) * dt for key, _ in limits]
            accept, bad, newdt, emax = rk12_rule(dt, errs, [lim for _, lim in limits], self.mindt, self.maxdt)
            self.dt = newdt
            self.last_err = emax
            if accept:
                self.y = ynew
                self.t = t0 + dt
                break
            if tr > 10:
                raise RuntimeError("The solver cannot converge after 10 badsteps")
            self.bad_steps += 1
            tr += 1
        self.step_count += 1

    def _eq_keys(self):
        return [k for k in ("m", "Te", "Tl") if k in self.y]

    def _am12(self):
        """solve_am01.go:45-318 (solver/am12): explicit Euler start, implicit Euler predictor and
        trapezoidal corrector solved by fixed-point iteration (target error 0.1 of the
        tolerance, at most 6 sweeps, divergence when alpha >= 1), error = predictor vs
        corrector in the am_error norm, dt_new = dt sqrt(0.8 / err) (limited by
        dt sqrt(0.6 / alpha) after a failed iteration, for the first equation only, as the
        reference resets the flag inside its loop), minimum over the equations.  m is
        renormalised where the reference's update renormalises it: before every right-hand
        side, so the iterators compare the renormalised previous iterate with the new raw one,
        and the final error compares the raw corrector and predictor results.  A failed
        iteration halves dt (or scales it by sqrt(0.6 / alpha) when alpha > 0.6) and retries
        without counting a bad step, as the reference does; 64 such retries in one step raise
        here (the reference keeps halving).  The thermal field is drawn per attempt."""
        f = self.model.rhs
        t0 = self.t
        keys = self._eq_keys()
        ab = [self.maxabserr[k] for k in keys]
        rl = [self.maxrelerr[k] for k in keys]
        y0 = self._fix(self.y)
        tries = 0
        aborts = 0
        restrict = False
        s_alpha = [0.0] * len(keys)
        while True:
            dt = self.dt
            self._thermal(dt)
            dy0 = f(t0, y0)
            y = self._fix(_comb(y0, [dy0], [1.0], dt))
            dy = f(t0 + dt, y)
            dybuf = dy
            failed = False
            for phase in ("predictor", "corrector"):
                er = [0.1] * len(keys)
                it = 0
                while True:
                    terrs = []
                    ynew = {}
                    for i, k in enumerate(keys):
                        if phase == "predictor":
                            ynew[k] = y0[k] + dt * dy[k]
                        else:
                            ynew[k] = y0[k] + 0.5 * dt * (dy[k] + dy0[k])
                        terrs.append(am_error(y[k], ynew[k], ynew[k], ab[i], rl[i]))
                    er, alp, err, alpha = am_iter_rule(er, terrs)
                    if phase == "predictor":
                        s_alpha = alp
                    y = dict(y, **ynew)
                    it += 1
                    self.iterations += 1
                    if err <= 0.1:
                        break
                    if alpha >= 1.0 or it > 5:
                        failed = True
                        break
                    y = self._fix(y)
                    dy = f(t0 + dt, y)
                if failed:
                    if tries == 9:
                        raise RuntimeError("The BDF iterator cannot converge")
                    h = 0.5 * dt
                    if alpha > 0.6:
                        h = dt * math.sqrt(0.6 / alpha)
                    self.dt = h
                    if phase == "predictor":
                        restrict = True
                    aborts += 1
                    if aborts > 64:
                        raise RuntimeError("am12: 64 failed iterations in one step")
                    break
                if phase == "predictor":
                    y1 = dict(y)
                    dy = dybuf
            if failed:
                continue
            bad = False
            ndts = []
            for i, k in enumerate(keys):
                terr = am_error(y[k], y1[k], y1[k], ab[i], rl[i])
                if terr > 1.0:
                    bad = True
                h_r = dt * math.sqrt(_div(0.8, terr))
                nd = h_r
                if restrict:
                    nd = min(h_r, dt * math.sqrt(_div(0.6, s_alpha[i])))
                    restrict = False
                nd = min(max(nd, self.mindt), self.maxdt)
                ndts.append(nd)
                self.last_err = max(self.last_err if i else 0.0, terr)
            ndt = min(ndts)
            self.dt = ndt
            if not bad or ndt == self.mindt:
                self.y = y
                self.t = t0 + dt
                break
            if tries > 10:
                raise RuntimeError("The solver cannot converge after 10 badsteps")
            self.bad_steps += 1
            tries += 1
        self.step_count += 1

    def _bdf_euler(self):
        """solve_euler_backward.go:29-91 (solver/bdf-euler, fixed step): time advanced first;
        each equation in turn (m, Te, Tl) takes an explicit Euler step and is then iterated,
        y = y0 + dt f(t + dt, y) with f evaluated on the current state of every equation,
        until MaxDiff(y, y_new) / MaxSum(y, y_new) <= max_iter_err; more than max_iter
        sweeps raise, as the reference panics.  m is renormalised before each evaluation."""
        f = self.model.rhs
        dt = self.dt
        self._thermal(dt)
        y = self._fix(self.y)
        dy = f(self.t, y)            # the inputs of the step, before time advances
        self.t += dt
        for k in self._eq_keys():
            y0k = y[k]
            y = dict(y)
            y[k] = y0k + dt * dy[k]
            y = self._fix(y)
            dy = f(self.t, y)
            self.iterations += 1
            it = 0
            err = 1.0e38
            while err > self.max_iter_err:
                ynew = y0k + dt * dy[k]
                err = float(np.abs(y[k] - ynew).max())
                ssum = float(np.abs(y[k] + ynew).max())
                if ssum > 0.0:
                    err = err / ssum
                it += 1
                self.iterations += 1
                y = dict(y)
                y[k] = ynew
                y = self._fix(y)
                dy = f(self.t, y)
                if it > self.max_iter:
                    raise RuntimeError("The BDF iterator cannot converge for %s" % k)
        self.y = y
        self.step_count += 1

    # -- new integrators ----------------------------------------------------------
    def _rk4(self):
        f, h, t = self.model.rhs, self.dt, self.t
        self._thermal(h)
        y0 = self.y
        k1 = f(t, y0)
        y2 = self._fix(_comb(y0, [k1], [0.5], h))
        k2 = f(t + 0.5 * h, y2)
        y3 = self._fix(_comb(y0, [k2], [0.5], h))
        k3 = f(t + 0.5 * h, y3)
        y4 = self._fix(_comb(y0, [k3], [1.0], h))
        k4 = f(t + h, y4)
        self.y = self._fix(_comb(y0, [k1, k2, k3, k4], [1 / 6, 1 / 3, 1 / 3, 1 / 6], h))
        self.t = t + h
        self.step_count += 1

    def _err_norm(self, y0, y1, e):
        err = 0.0
        for key in e:
            d = np.abs(e[key])
            if key == "m":
                v = float(d.max()) / self.rtol
            else:
                scale = self.rtol * np.maximum(np.abs(y0[key]), np.abs(y1[key]))
                v = float((d / np.where(scale == 0.0, 1.0, scale)).max())
            err = max(err, v)
        return err

    def _dp45(self):
        f, t0 = self.model.rhs, self.t
        y0 = self.y
        if self.k_fsal is None:
            self._thermal(self.dt)
            self.k_fsal = f(t0, y0)
        for tr in range(64):
            h = self.dt
            self._thermal(h)
            if self.model.s.thermal:
                # the held thermal field changes with the step (and its dt), so the
                # first stage is re-evaluated instead of reusing the last one
                self.k_fsal = f(t0, y0)
            ks = [self.k_fsal]
            for s in range(1, 7):
                ys = self._fix(_comb(y0, ks, DP_A[s], h))
                ks.append(f(t0 + DP_C[s] * h, ys))
            y5 = ys
            e = {key: h * sum(DP_E[i] * ks[i][key] for i in range(7)) for key in y0}
            err = self._err_norm(y0, y5, e)
            self.last_err = err
            accept = err <= 1.0 or h <= self.mindt
            if err == 0.0:
                fac = 5.0
            else:
                fac = 0.9 * err ** -0.2
            fac = min(max(fac, 0.2), 5.0 if accept else 1.0)
            self.dt = min(max(h * fac, self.mindt), self.maxdt)
            if accept:
                self.y = y5
                self.t = t0 + h
                self.k_fsal = ks[6]
                break
            self.bad_steps += 1
        self.step_count += 1
