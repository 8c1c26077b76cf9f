"""Continuous-batching request loop over size-class batches (``hsb_batch_*``).

hotspin runs one simulation per process (``engine/engine.go``); serving many independent
LLG/LLB solves on one GPU is new here.  Requests arrive over time; each belongs to a size
class (grid size, boundaries, solver and tolerance, channel count, demag, thermal field).
A class is one ``Batch``: up to ``nslot`` slots advanced together by the same kernels and
one captured CUDA graph per class, on its own stream, so classes overlap on the GPU.  Each
slot has its own physics, cell size and demag kernel.  The loop

* admits arrived requests into free slots of their class, creating the class when the
  device-memory budget (``Batch.footprint``: state arenas, RK stages, demag spectra and plan)
  allows, and evicting idle classes when it does not;
* relaunches every class whose previous launch finished, and never waits for a class that
  is still running;
* collects each request when its slot reports its end time reached, and frees the slot
  for the next request at once (continuous batching, not a queue of fixed batches).

Results of a request do not depend on what else is in flight: every kernel touches only
its own slot's arena and solver word.
"""
import collections
import dataclasses
import math
import time

import numpy as np

from .sim import Batch, Simulation

MU0 = 4.0e-7 * math.pi
MUB = 9.27400968202020202e-24


@dataclasses.dataclass
class Request:
    rid: int
    desc: dict            # Simulation / Batch.admit keywords (program order)
    m0: np.ndarray        # (3, N0, N1, N2) float64
    t_end: float          # simulated end time (s)
    arrival: float = 0.0  # seconds after the start of the run

    @property
    def ncell(self):
        s = self.desc["size"]
        return int(s[0] * s[1] * s[2])


@dataclasses.dataclass
class Result:
    rid: int
    m: np.ndarray
    steps: int
    attempts: int
    t: float
    status: int
    arrival: float
    admitted: float
    done: float

    @property
    def time_to_solution(self):
        return self.done - self.arrival


CLASS_KEYS = ("size", "pbc", "solver", "rtol", "ttm", "demag", "thermal")


def class_key(desc):
    """Size-class key: what one batch must share."""
    vals = []
    for k in CLASS_KEYS:
        v = desc.get(k, 0)
        vals.append(tuple(v) if isinstance(v, (list, tuple)) else v)
    return tuple(vals)


def class_desc(desc):
    """Class-wide descriptor fields of a request (what ``Batch`` is created with)."""
    return {k: desc[k] for k in ("size", "pbc", "cellsize", "solver", "rtol", "ttm", "demag", "thermal", "dt",
                                 "msat0T0", "gamma_ll") if k in desc}


class _Class:
    def __init__(self, key, batch, footprint):
        self.key = key
        self.batch = batch
        self.footprint = footprint
        self.free = list(range(batch.nslot - 1, -1, -1))
        self.occupant = {}        # slot -> (Request, admitted time)
        self.busy = False
        self.launches = 0

    @property
    def idle(self):
        return not self.occupant and not self.busy


class Server:
    """Continuous-batching loop.

    hbm_budget: device bytes the batches may hold together (admission by footprint).
    cells_per_class: slots of a class = clamp(cells_per_class // ncell, 1, max_slots).
    graphs_per_launch: class-graph launches between two looks at a class's slots.
    """

    def __init__(self, hbm_budget=32 << 30, cells_per_class=1 << 21, max_slots=64, graphs_per_launch=1):
        self.hbm_budget = int(hbm_budget)
        self.cells_per_class = int(cells_per_class)
        self.max_slots = int(max_slots)
        self.graphs_per_launch = int(graphs_per_launch)
        self.classes = {}
        self.used = 0
        self.stats = collections.Counter()

    def slots_for(self, ncell):
        return max(1, min(self.max_slots, self.cells_per_class // max(1, ncell)))

    # ---------------------------------------------------------------- classes
    def _open_class(self, req):
        key = class_key(req.desc)
        cdesc = class_desc(req.desc)
        nslot = self.slots_for(req.ncell)
        need = Batch.footprint(nslot, **cdesc)
        while nslot > 1 and need > self.hbm_budget:
            nslot = max(1, nslot // 2)
            need = Batch.footprint(nslot, **cdesc)
        if need > self.hbm_budget:
            raise ValueError("request %d needs %d device bytes, above the budget of %d"
                             % (req.rid, need, self.hbm_budget))
        if self.used + need > self.hbm_budget:
            for k in [k for k, c in self.classes.items() if c.idle]:
                self._close_class(k)
                if self.used + need <= self.hbm_budget:
                    break
        if self.used + need > self.hbm_budget:
            self.stats["deferred_by_footprint"] += 1
            return None
        c = _Class(key, Batch(nslot, **cdesc), need)
        self.classes[key] = c
        self.used += need
        self.stats["classes_opened"] += 1
        return c

    def _close_class(self, key):
        c = self.classes.pop(key)
        c.batch.close()
        self.used -= c.footprint

    def close(self):
        for k in list(self.classes):
            self._close_class(k)

    # ---------------------------------------------------------------- loop
    def run(self, requests, realtime=True, clock=time.perf_counter):
        """Serve `requests` (arrival offsets in seconds); returns {rid: Result}.

        realtime: requests become visible at their arrival offsets after the start; when
        False every request is available at once.
        """
        order = sorted(requests, key=lambda r: r.arrival)
        pending = collections.deque(order)
        waiting = collections.OrderedDict()     # key -> deque of requests
        results = {}
        t0 = clock()
        total = len(order)
        while len(results) < total:
            now = clock() - t0
            while pending and (not realtime or pending[0].arrival <= now):
                r = pending.popleft()
                waiting.setdefault(class_key(r.desc), collections.deque()).append(r)
            progressed = False
            for key in list(self.classes):
                c = self.classes[key]
                if c.busy:
                    if not c.batch.poll():
                        continue
                    c.busy = False
                    progressed = True
                    self._collect(c, results, t0, clock)
                self._admit(c, waiting.get(key), clock() - t0)
                if c.occupant:
                    c.batch.launch(self.graphs_per_launch)
                    c.busy = True
                    c.launches += 1
            # classes for waiting requests that have none yet
            for key, q in list(waiting.items()):
                if q and key not in self.classes:
                    c = self._open_class(q[0])
                    if c is not None:
                        self._admit(c, q, clock() - t0)
                        c.batch.launch(self.graphs_per_launch)
                        c.busy = True
                        c.launches += 1
                        progressed = True
                if not q:
                    waiting.pop(key, None)
            if not progressed and not any(c.busy for c in self.classes.values()):
                if pending and realtime:
                    time.sleep(max(0.0, min(0.002, pending[0].arrival - (clock() - t0))))
                elif not pending and not any(waiting.values()):
                    break
        return results

    def _admit(self, c, q, now):
        while q and c.free:
            r = q.popleft()
            slot = c.free.pop()
            c.batch.admit(slot, r.m0, r.t_end, **r.desc)
            c.occupant[slot] = (r, now)
            self.stats["admitted"] += 1

    def _collect(self, c, results, t0, clock):
        for slot in list(c.occupant):
            st = c.batch.slot_status(slot)
            if st["active"]:
                continue
            r, adm = c.occupant.pop(slot)
            m = c.batch.slot_get(slot, "m")
            results[r.rid] = Result(r.rid, m, st["steps"], st["attempts"], st["t"], st["status"], r.arrival, adm,
                                    clock() - t0)
            c.free.append(slot)


def run_sequential(requests, clock=time.perf_counter):
    """The plain path: one Simulation per request, in arrival order, one at a time.

    Service times are measured; a request starts at max(its arrival, the previous
    completion), as on a server that runs them back to back.  Returns ({rid: Result},
    {rid: service seconds}, {rid: setup seconds}).
    """
    results, service, setup = {}, {}, {}
    free_at = 0.0
    for r in sorted(requests, key=lambda q: q.arrival):
        a = clock()
        sim = Simulation(**r.desc)
        sim.set("m", r.m0)
        b = clock()
        sim.run_until(r.t_end)
        m = sim.get("m")
        st = sim.status()
        sim.close()
        e = clock()
        start = max(r.arrival, free_at)
        free_at = start + (e - a)
        service[r.rid] = e - a
        setup[r.rid] = b - a
        results[r.rid] = Result(r.rid, m, st["steps"], st["attempts"], st["t"], st["status"], r.arrival, start,
                                free_at)
    return results, service, setup


# -------------------------------------------------------------------- synthetic request stream
def equilibrium_m_half(T, Tc):
    """Mean-field m_e(T) for J = 1/2 (m = tanh(m Tc / T)), by bisection."""
    if T <= 0:
        return 1.0
    if T >= Tc:
        return 0.0
    lo, hi = 1e-12, 1.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if math.tanh(mid * Tc / T) > mid:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def make_requests(n=256, rate=50.0, seed=4, t_end=50e-12, sides=(32, 64, 128, 256, 512), layers=(1, 2),
                  llb_min_T=300.0, tc=630.0, a_ex=1.3e-11, rtol=1e-5):
    """Poisson stream of independent LLG/LLB requests with seeded parameters.

    Square films with a side drawn log-uniformly from `sides` and 1 or 2 layers; cubic
    cells of 2-5 nm; Ms0 4e5-1.2e6 A/m; damping 0.005-0.1; T 0-600 K; a seeded random
    initial m; a 0-50 mT field in a random direction; DP45 at `rtol` to `t_end`.
    Requests below `llb_min_T` run as LLG (|m| = 1, Brown thermal field at T): the MFA
    longitudinal relaxation of LLB gets too stiff for an explicit integrator at low T
    (its rate grows like 1/chi_par(T), > 1e16 /s below about 100 K at Tc = 630 K).  Above
    it they run as LLB (J = 1/2, Tc = `tc`) with m starting at length m_e(T).
    """
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        side = int(sides[rng.integers(len(sides))])
        nz = int(layers[rng.integers(len(layers))])
        size = (nz, side, side)
        cs = float(rng.uniform(2e-9, 5e-9))
        ms = float(rng.uniform(4e5, 1.2e6))
        alpha = float(rng.uniform(0.005, 0.1))
        T = float(rng.uniform(0.0, 600.0))
        bmag = float(rng.uniform(0.0, 0.05))
        bdir = rng.normal(size=3)
        bdir /= np.linalg.norm(bdir)
        m0 = rng.normal(size=(3,) + size)
        m0 /= np.sqrt((m0 * m0).sum(0))
        llb = T >= llb_min_T
        if llb:
            m0 *= equilibrium_m_half(T, tc)
        lex = math.sqrt(2.0 * a_ex / (MU0 * ms * ms))
        desc = dict(size=size, cellsize=(cs, cs, cs), pbc=(0, 0, 0), msat0T0=ms, lex=lex,
                    alpha=(alpha, alpha, alpha), b_ext=tuple(float(x) for x in bmag * bdir),
                    demag=True, normalize=not llb, llb=llb, tc=tc, spin_j=0.5,
                    n_spins=ms / (2 * MUB * 0.5), temperature=T, thermal=T > 0.0, seed=1000 + i,
                    solver="dp45", dt=1e-15, rtol=rtol, mindt=1e-22, maxdt=1e-12)
        reqs.append(Request(i, desc, m0, t_end, t))
    return reqs


def summarize(results, requests):
    """p50/p99 time-to-solution, throughput (requests/s, Mcell-steps/s) over the makespan."""
    byid = {r.rid: r for r in requests}
    tts = np.array([res.time_to_solution for res in results.values()])
    first = min(r.arrival for r in requests)
    last = max(res.done for res in results.values())
    span = last - first
    cell_steps = sum(byid[k].ncell * res.steps for k, res in results.items())
    return dict(n=len(results), p50_s=float(np.percentile(tts, 50)), p99_s=float(np.percentile(tts, 99)),
                makespan_s=span, req_per_s=len(results) / span, mcell_steps_per_s=cell_steps / span / 1e6,
                steps_mean=float(np.mean([res.steps for res in results.values()])))
