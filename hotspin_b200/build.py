"""Build libhsb200.so (in-tree) from hotspin_b200/csrc with nvcc for sm_100a.

    python -m hotspin_b200.build [--force]

Objects go to hotspin_b200/_build/, the library to hotspin_b200/libhsb200.so.  Kernel_Arne
(hsb_arne.cu) is compiled without FMA contraction so its FP64 sums round like the
sequential reference code.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libhsb200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                 "-I" + SRC, "-I" + os.path.join(os.path.dirname(HERE), "include")]
PER_FILE = {"hsb_arne.cu": ["-fmad=false"]}


def sources():
    return sorted(f for f in os.listdir(SRC) if f.endswith(".cu"))


def _newest_header():
    hs = [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".cuh", ".h"))]
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src, force):
    s = os.path.join(SRC, src)
    o = os.path.join(OBJ, src[:-3] + ".o")
    if not force and os.path.exists(o) and os.path.getmtime(o) >= max(os.path.getmtime(s), _newest_header()):
        return o, None
    cmd = [NVCC] + COMMON + PER_FILE.get(src, []) + ["-c", s, "-o", o]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        return o, "%s\n%s\n%s" % (" ".join(cmd), p.stdout, p.stderr)
    return o, None


def build(force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    srcs = sources()
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        results = list(ex.map(lambda s: _compile(s, force), srcs))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    tmp = LIB + ".tmp%d" % os.getpid()
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s\n%s" % (" ".join(cmd), p.stdout, p.stderr))
    os.replace(tmp, LIB)
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
