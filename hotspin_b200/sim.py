"""Python view of the simulation handle (hsb_sim_* in include/hotspin_b200.h).

Arrays are numpy float64 in hotspin's program order: scalar fields (N0, N1, N2), vector
fields (3, N0, N1, N2) with component 0 the program X axis (user z).
"""
import ctypes

import numpy as np

from . import _lib

SOLVERS = {"euler": 0, "heun": 1, "rk4": 2, "dp45": 3, "rk45": 3, "rk12": 4, "am12": 5, "bdf-euler": 6,
           "bdf_euler": 6}

_FIELDS = {f[0] for f in _lib.SimDesc._fields_}


def make_desc(**kw):
    """Build an hsb_sim_desc from keyword arguments (names as in the C struct)."""
    d = _lib.SimDesc()
    d.gamma_ll = 2.211e5
    d.spin_j = 0.5
    d.rtol = 1e-5
    d.mindt = 1e-22
    d.maxdt = 1e-12
    d.laser_fwhm = 1e-13
    for k, v in kw.items():
        if k == "laser_table":
            # pointwise laser time profile: (t, factor) pairs, copied by hsb_sim_create
            tab = np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(-1, 2))
            d._laser_keep = tab          # alive as long as the descriptor
            d.laser_table = tab.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            d.laser_npts = tab.shape[0]
            continue
        if k == "bext_table":
            # pointwise applied field: (t, Bx, By, Bz) rows in tesla, program components
            tab = np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(-1, 4))
            d._bext_keep = tab
            d.bext_table = tab.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            d.bext_npts = tab.shape[0]
            continue
        if k not in _FIELDS or k in ("laser_npts", "bext_npts"):
            raise KeyError("unknown simulation parameter %r" % k)
        if k == "solver" and isinstance(v, str):
            v = SOLVERS[v.lower()]
        if k == "demag_tensor" and isinstance(v, str):
            v = DEMAG_TENSORS[v.lower()]
        cur = getattr(d, k)
        if isinstance(cur, ctypes.Array):
            for i, x in enumerate(v):
                cur[i] = x
        elif isinstance(v, bool):
            setattr(d, k, int(v))
        else:
            setattr(d, k, v)
    return d


class Simulation:
    def __init__(self, **kw):
        self._lib = _lib.load()
        self.desc = make_desc(**kw)
        self.size = tuple(self.desc.size)
        self.ncell = int(np.prod(self.size))
        h = ctypes.c_void_p()
        _lib.check(self._lib.hsb_sim_create(ctypes.byref(self.desc), ctypes.byref(h)), "hsb_sim_create")
        self._h = h

    # -- lifetime
    def close(self):
        if getattr(self, "_h", None):
            self._lib.hsb_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- state
    def set(self, name, arr):
        if arr is None:
            _lib.check(self._lib.hsb_sim_set(self._h, name.encode(), None, 0), "hsb_sim_set(%s)" % name)
            return
        a = np.ascontiguousarray(arr, dtype=np.float64)
        _lib.check(self._lib.hsb_sim_set(self._h, name.encode(), a.ctypes.data_as(_lib.c_dp), a.size),
                   "hsb_sim_set(%s)" % name)

    def get(self, name, out=None):
        """The quantity as a new float64 array, or written into ``out`` (C-contiguous float64
        of the quantity's shape, e.g. a view of page-locked host memory)."""
        ncomp = {"m": 3, "H_demag": 3, "Te": 1, "Tl": 1}.get(name)
        if name == "k":
            ncomp = 5 if self.desc.ttm else 3
        if ncomp is None:
            raise KeyError(name)
        shape = (ncomp,) + self.size if ncomp > 1 else self.size
        if out is None:
            out = np.empty(shape, dtype=np.float64)
        elif out.shape != shape or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("out must be C-contiguous float64 of shape %s" % (shape,))
        _lib.check(self._lib.hsb_sim_get(self._h, name.encode(), out.ctypes.data_as(_lib.c_dp), out.size),
                   "hsb_sim_get(%s)" % name)
        return out

    # -- time stepping
    def step(self, n=1):
        _lib.check(self._lib.hsb_sim_step(self._h, int(n)), "hsb_sim_step")

    def run_until(self, t):
        _lib.check(self._lib.hsb_sim_run_until(self._h, float(t)), "hsb_sim_run_until")

    def sync(self):
        _lib.check(self._lib.hsb_sim_sync(self._h), "hsb_sim_sync")

    def status(self):
        t, dt, err = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        st, at, rj = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        s = ctypes.c_int32()
        _lib.check(self._lib.hsb_sim_status(self._h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(st),
                                            ctypes.byref(at), ctypes.byref(rj), ctypes.byref(err),
                                            ctypes.byref(s)), "hsb_sim_status")
        return dict(t=t.value, dt=dt.value, steps=st.value, attempts=at.value, rejects=rj.value,
                    err=err.value, status=s.value)

    def set_time(self, t, dt=0.0):
        _lib.check(self._lib.hsb_sim_set_time(self._h, float(t), float(dt)), "hsb_sim_set_time")

    def energy(self):
        e = ctypes.c_double()
        _lib.check(self._lib.hsb_sim_energy(self._h, ctypes.byref(e)), "hsb_sim_energy")
        return e.value

    def energy_terms(self):
        """Zeeman, exchange, demag, anisotropy and longitudinal-field energies (J)."""
        a = (ctypes.c_double * 5)()
        _lib.check(self._lib.hsb_sim_energy_terms(self._h, a), "hsb_sim_energy_terms")
        return dict(zip(("zeeman", "exchange", "demag", "anisotropy", "longitudinal"), list(a)))

    def average_m(self):
        a = (ctypes.c_double * 3)()
        _lib.check(self._lib.hsb_sim_average_m(self._h, a), "hsb_sim_average_m")
        return np.array(list(a))

    def checkpoint(self):
        """Keep the current state and solver position on the device (see restore)."""
        _lib.check(self._lib.hsb_sim_checkpoint(self._h), "hsb_sim_checkpoint")

    def restore(self):
        """Return to the last checkpoint; stepping then repeats the original continuation."""
        _lib.check(self._lib.hsb_sim_restore(self._h), "hsb_sim_restore")

    def launch_count(self):
        """Kernels the handle has enqueued for stepping since creation."""
        n = ctypes.c_int64()
        _lib.check(self._lib.hsb_sim_launch_count(self._h, ctypes.byref(n)), "hsb_sim_launch_count")
        return n.value

    def max_torque(self):
        """max over cells of |gamma (m x H_eff)| (1/s), reduced on the device."""
        v = ctypes.c_double()
        _lib.check(self._lib.hsb_sim_max_torque(self._h, ctypes.byref(v)), "hsb_sim_max_torque")
        return v.value


class Batch:
    """A size class of simulations advanced together (hsb_batch_* in include/hotspin_b200.h).

    ``cls`` holds the class-wide descriptor fields (size, pbc, solver, rtol, demag, ttm,
    thermal; plus valid defaults for the rest); slots are loaded with ``admit``, each with its
    own descriptor (cell size and demag kernel included).
    """

    def __init__(self, nslot, **cls):
        self._lib = _lib.load()
        self.desc = make_desc(**cls)
        self.size = tuple(self.desc.size)
        self.ncell = int(np.prod(self.size))
        h = ctypes.c_void_p()
        _lib.check(self._lib.hsb_batch_create(ctypes.byref(self.desc), int(nslot), ctypes.byref(h)),
                   "hsb_batch_create")
        self._h = h
        ns, ap, nc = _lib.c_i32(), _lib.c_i32(), _lib.c_i64()
        _lib.check(self._lib.hsb_batch_info(h, ctypes.byref(ns), ctypes.byref(ap), ctypes.byref(nc)),
                   "hsb_batch_info")
        self.nslot, self.attempts_per_graph = ns.value, ap.value

    @staticmethod
    def footprint(nslot, **cls):
        lib = _lib.load()
        d = make_desc(**cls)
        b = _lib.c_i64()
        _lib.check(lib.hsb_batch_footprint(ctypes.byref(d), int(nslot), ctypes.byref(b)), "hsb_batch_footprint")
        return b.value

    def close(self):
        if getattr(self, "_h", None):
            self._lib.hsb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def admit(self, slot, m, t_stop, **kw):
        """Load a simulation (descriptor keywords as for Simulation) with initial m into `slot`."""
        d = make_desc(**kw)
        a = np.ascontiguousarray(m, dtype=np.float64)
        if a.size != 3 * self.ncell:
            raise ValueError("m must hold 3 x %d values" % self.ncell)
        _lib.check(self._lib.hsb_batch_admit(self._h, int(slot), ctypes.byref(d), a.ctypes.data_as(_lib.c_dp),
                                             float(t_stop)), "hsb_batch_admit")

    def launch(self, graphs=1):
        _lib.check(self._lib.hsb_batch_launch(self._h, int(graphs)), "hsb_batch_launch")

    def poll(self):
        d = _lib.c_i32()
        _lib.check(self._lib.hsb_batch_poll(self._h, ctypes.byref(d)), "hsb_batch_poll")
        return bool(d.value)

    def slot_status(self, slot):
        t, dt = ctypes.c_double(), ctypes.c_double()
        st, at, rj = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        s, a = ctypes.c_int32(), ctypes.c_int32()
        _lib.check(self._lib.hsb_batch_slot_status(self._h, int(slot), ctypes.byref(t), ctypes.byref(dt),
                                                   ctypes.byref(st), ctypes.byref(at), ctypes.byref(rj),
                                                   ctypes.byref(s), ctypes.byref(a)), "hsb_batch_slot_status")
        return dict(t=t.value, dt=dt.value, steps=st.value, attempts=at.value, rejects=rj.value,
                    status=s.value, active=bool(a.value))

    def slot_get(self, slot, name="m"):
        ncomp = {"m": 3, "Te": 1, "Tl": 1}[name]
        out = np.empty((ncomp,) + self.size if ncomp > 1 else self.size, dtype=np.float64)
        _lib.check(self._lib.hsb_batch_slot_get(self._h, int(slot), name.encode(), out.ctypes.data_as(_lib.c_dp),
                                                out.size), "hsb_batch_slot_get(%s)" % name)
        return out

    def release(self, slot):
        _lib.check(self._lib.hsb_batch_release(self._h, int(slot)), "hsb_batch_release")


DEMAG_TENSORS = {"arne": 0, "newell": 1}


def demag_plan(size, cellsize, pbc=(0, 0, 0), accuracy=6, stream=None, tensor="arne"):
    """Create a demag plan; returns an opaque handle (ctypes.c_void_p).  tensor: "arne"
    (hotspin's Kernel_Arne) or "newell" (the closed-form FP64 Newell tensor)."""
    lib = _lib.load()
    h = ctypes.c_void_p()
    s = (ctypes.c_int * 3)(*size)
    c = (ctypes.c_double * 3)(*cellsize)
    p = (ctypes.c_int * 3)(*pbc)
    _lib.check(lib.hsb_demag_plan_create_tensor(s, c, p, accuracy, DEMAG_TENSORS[tensor], stream, ctypes.byref(h)),
               "hsb_demag_plan_create")
    return h
