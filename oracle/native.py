"""Build and load the oracle's C restatements (test infrastructure only).

``oracle/csrc/*.c`` is compiled with gcc into ``oracle/_build/liboracle.so`` (OpenMP, no
fast-math, no FMA contraction so the arithmetic order of the restated Go code is kept).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "csrc")
_OUT = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build(force=False):
    srcs = sorted(os.path.join(_SRC, f) for f in os.listdir(_SRC) if f.endswith(".c"))
    newest = max(os.path.getmtime(s) for s in srcs)
    if not force and os.path.exists(_OUT) and os.path.getmtime(_OUT) >= newest:
        return _OUT
    os.makedirs(os.path.dirname(_OUT), exist_ok=True)
    tmp = _OUT + ".tmp%d" % os.getpid()
    cmd = ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", "-o", tmp] + srcs + ["-lm"]
    subprocess.check_call(cmd)
    os.replace(tmp, _OUT)
    return _OUT


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        _lib.hsb_oracle_kernel_arne.argtypes = [ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(ctypes.c_double),
                                               ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                               ctypes.POINTER(ctypes.c_double)]
        _lib.hsb_oracle_kernel_arne.restype = ctypes.c_int
    return _lib


def kernel_arne(size, cellsize, pbc, accuracy=6):
    """C restatement of Kernel_Arne; same result as ``oracle.demag.kernel_arne``."""
    size = [int(s) for s in size]
    K = np.zeros((6,) + tuple(size), dtype=np.float64)
    s = (ctypes.c_int * 3)(*size)
    c = (ctypes.c_double * 3)(*[float(x) for x in cellsize])
    p = (ctypes.c_int * 3)(*[int(x) for x in pbc])
    rc = lib().hsb_oracle_kernel_arne(s, c, p, int(accuracy),
                                     K.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    if rc != 0:
        raise RuntimeError("kernel_arne failed")
    return K
