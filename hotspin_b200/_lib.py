"""ctypes binding of libhsb200.so.

The library is built in-tree by ``hotspin_b200.build``.  There is no CPU fallback: if the
shared library is missing or cannot be loaded, every entry point raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhsb200.so")

_lib = None

c_int = ctypes.c_int
c_i32 = ctypes.c_int32
c_i64 = ctypes.c_int64
c_u64 = ctypes.c_uint64
c_dbl = ctypes.c_double
c_vp = ctypes.c_void_p
c_dp = ctypes.POINTER(ctypes.c_double)
c_ip = ctypes.POINTER(ctypes.c_int)


class HsbError(RuntimeError):
    pass


class SimDesc(ctypes.Structure):
    """Mirror of hsb_sim_desc (include/hotspin_b200.h)."""
    _fields_ = [
        ("size", c_i32 * 3), ("pbc", c_i32 * 3), ("cellsize", c_dbl * 3),
        ("msat0T0", c_dbl), ("lex", c_dbl), ("gamma_ll", c_dbl), ("alpha", c_dbl * 3),
        ("ku", c_dbl), ("anis_u", c_dbl * 3), ("b_ext", c_dbl * 3),
        ("demag", c_i32), ("normalize", c_i32), ("llb", c_i32),
        ("tc", c_dbl), ("spin_j", c_dbl), ("n_spins", c_dbl), ("temperature", c_dbl),
        ("thermal", c_i32), ("seed", c_u64), ("cutoff_dt", c_dbl),
        ("ttm", c_i32), ("gamma_e", c_dbl), ("c_l", c_dbl), ("g_ep", c_dbl), ("k_e", c_dbl),
        ("k_l", c_dbl), ("laser_p0", c_dbl), ("laser_t0", c_dbl), ("laser_fwhm", c_dbl),
        ("laser_sigma", c_dbl), ("solver", c_i32), ("dt", c_dbl), ("rtol", c_dbl),
        ("mindt", c_dbl), ("maxdt", c_dbl), ("laser_table", ctypes.POINTER(c_dbl)), ("laser_npts", c_i32),
        ("bext_table", ctypes.POINTER(c_dbl)), ("bext_npts", c_i32), ("maxerr", c_dbl * 3),
        ("maxrelerr", c_dbl * 3), ("max_iter", c_i32), ("demag_tensor", c_i32),
        ("mu_par", c_dbl * 3), ("mu_perp", c_dbl * 3), ("alpha_e", c_dbl * 3),
    ]


# exported symbol -> (restype, argtypes); drop-ins return void
_SIGS = {
    "hsb_last_error": (ctypes.c_char_p, []),
    "hsb_clear_error": (None, []),
    "hsb_version": (c_int, []),
    "hsb_sim_desc_bytes": (c_int, []),
    "hsb_solver_word_bytes": (c_int, []),
    "hsb_crc64_iso": (ctypes.c_uint64, [c_vp, ctypes.c_int64]),
    "hsb_sim_create": (c_int, [ctypes.POINTER(SimDesc), ctypes.POINTER(c_vp)]),
    "hsb_sim_destroy": (c_int, [c_vp]),
    "hsb_sim_set": (c_int, [c_vp, ctypes.c_char_p, c_dp, c_i64]),
    "hsb_sim_get": (c_int, [c_vp, ctypes.c_char_p, c_dp, c_i64]),
    "hsb_sim_set_device": (c_int, [c_vp, ctypes.c_char_p, c_vp, c_i64]),
    "hsb_sim_get_device": (c_int, [c_vp, ctypes.c_char_p, c_vp, c_i64]),
    "hsb_sim_step": (c_int, [c_vp, c_i64]),
    "hsb_sim_run_until": (c_int, [c_vp, c_dbl]),
    "hsb_sim_sync": (c_int, [c_vp]),
    "hsb_sim_status": (c_int, [c_vp, c_dp, c_dp, ctypes.POINTER(c_i64), ctypes.POINTER(c_i64),
                               ctypes.POINTER(c_i64), c_dp, ctypes.POINTER(c_i32)]),
    "hsb_sim_set_time": (c_int, [c_vp, c_dbl, c_dbl]),
    "hsb_sim_energy": (c_int, [c_vp, c_dp]),
    "hsb_sim_average_m": (c_int, [c_vp, c_dp]),
    "hsb_sim_energy_terms": (c_int, [c_vp, c_dp]),
    "hsb_sim_max_torque": (c_int, [c_vp, c_dp]),
    "hsb_sim_stream": (c_vp, [c_vp]),
    "hsb_sim_profile": (c_int, [c_vp, c_int, c_dp]),
    "hsb_sim_launches_per_attempt": (c_int, [c_vp, c_ip]),
    "hsb_sim_launch_count": (c_int, [c_vp, ctypes.POINTER(c_i64)]),
    "hsb_sim_checkpoint": (c_int, [c_vp]),
    "hsb_sim_restore": (c_int, [c_vp]),
    "hsb_average_m_noalloc": (c_int, [c_vp, c_i64, c_vp, c_vp]),
    "hsb_set_stage_variant": (c_int, [c_int]),
    "hsb_stage_variant_of": (c_int, [c_vp]),
    "hsb_batch_footprint": (c_int, [ctypes.POINTER(SimDesc), c_i32, ctypes.POINTER(c_i64)]),
    "hsb_batch_create": (c_int, [ctypes.POINTER(SimDesc), c_i32, ctypes.POINTER(c_vp)]),
    "hsb_batch_destroy": (c_int, [c_vp]),
    "hsb_batch_info": (c_int, [c_vp, ctypes.POINTER(c_i32), ctypes.POINTER(c_i32), ctypes.POINTER(c_i64)]),
    "hsb_batch_admit": (c_int, [c_vp, c_i32, ctypes.POINTER(SimDesc), c_dp, c_dbl]),
    "hsb_batch_launch": (c_int, [c_vp, c_i32]),
    "hsb_batch_poll": (c_int, [c_vp, ctypes.POINTER(c_i32)]),
    "hsb_batch_slot_status": (c_int, [c_vp, c_i32, c_dp, c_dp, ctypes.POINTER(c_i64), ctypes.POINTER(c_i64),
                                      ctypes.POINTER(c_i64), ctypes.POINTER(c_i32), ctypes.POINTER(c_i32)]),
    "hsb_batch_slot_get": (c_int, [c_vp, c_i32, ctypes.c_char_p, c_dp, c_i64]),
    "hsb_batch_release": (c_int, [c_vp, c_i32]),
    "hsb_mfa_table": (c_int, [c_dbl, c_dbl, c_int, c_dp, c_dp, c_dp]),
    "hsb_mfa_equilibrium": (c_int, [c_dbl, c_dbl, c_dbl, c_dp]),
    "hsb_demag_profile": (c_int, [c_vp, c_vp, c_vp, c_dbl, c_vp, c_vp, c_int, c_dp]),
    "hsb_demag_plan_create_tensor": (c_int, [c_ip, c_dp, c_ip, c_int, c_int, c_vp, ctypes.POINTER(c_vp)]),
    "hsb_demag_plan_create": (c_int, [c_ip, c_dp, c_ip, c_int, c_vp, ctypes.POINTER(c_vp)]),
    "hsb_demag_plan_destroy": (c_int, [c_vp]),
    "hsb_demag_plan_info": (c_int, [c_vp, c_ip, c_ip, c_dp]),
    "hsb_demag_field": (c_int, [c_vp, c_vp, c_vp, c_dbl, c_vp, c_vp]),
    "hsb_demag_kernel_copy": (c_int, [c_vp, ctypes.POINTER(ctypes.c_float), ctypes.c_long]),
    "hsb_fft_plan_create": (c_int, [c_ip, c_ip, c_vp, ctypes.POINTER(c_vp)]),
    "hsb_fft_forward": (c_int, [c_vp, c_vp, c_vp]),
    "hsb_fft_inverse": (c_int, [c_vp, c_vp, c_vp]),
    "hsb_fft_plan_destroy": (c_int, [c_vp]),
}


def load():
    """Load libhsb200.so; raises HsbError when it is absent (no fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise HsbError("libhsb200.so not built: run `python -m hotspin_b200.build` (%s)" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(rc, what=""):
    if rc != 0:
        msg = load().hsb_last_error().decode(errors="replace")
        raise HsbError("%s failed (status %d): %s" % (what, rc, msg))


def exported_symbols_from_headers():
    """Every function name declared in include/*.h (used by the ABI tests)."""
    import re
    inc = os.path.join(os.path.dirname(HERE), "include")
    names = set()
    for f in sorted(os.listdir(inc)):
        if not f.endswith(".h"):
            continue
        txt = open(os.path.join(inc, f)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        txt = re.sub(r"//[^\n]*", "", txt)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", txt):
            name = m.group(1)
            pre = txt[max(0, m.start() - 80):m.start()]
            if name in ("if", "while", "for", "switch", "return", "sizeof", "defined"):
                continue
            if re.search(r"(typedef|#define)[^\n;]*$", pre):
                continue
            if re.search(r"\b(void|int|double|float|char|hsb_sim|hsb_batch|hsb_demag_plan)\s*\**\s*$", pre):
                names.add(name)
    return names
