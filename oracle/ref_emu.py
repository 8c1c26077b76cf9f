"""The reference's CUDA kernel library built for the CPU emulation of CUDA -- TEST INFRASTRUCTURE.

Compiles the reference checkout's ``src/libhotspin/*.cu`` and ``*.cpp`` (``$HOTSPIN_REF``,
default /root/reference) with the rewrites of ``tests/emu/build.py`` against the emulated
runtime of ``tests/emu`` into ``oracle/_ref/libhotspin_emu.so``.  With it the replay of
hotspin's call sequence (``oracle/replay.py``) runs the reference's own kernels on a machine
without a GPU, so the tests that compare the product with those kernels can run under
``pytest --emulate-cuda --emulate-reference``.

The reference's block reductions (reduce.cu) finish their last 32 values warp-synchronously:
no barrier, relying on the lanes of a warp executing in lockstep.  The emulation runs the
threads of a block one after another between barriers, which gives those reductions a wrong
result in the forward order; in reverse order (HSBEMU_ORDER=reverse, lane 31 first) every lane
reads the finished values of the higher lanes, a superset of what it reads in lockstep, which
gives the right result for the max reductions the replay uses (partialMaxAbs / partialMaxDiff)
but not for sums.  Tests on the emulated reference library therefore run in reverse order.

    python oracle/ref_emu.py
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_ROOT = os.environ.get("HOTSPIN_REF", "/root/reference")
OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT, "libhotspin_emu.so")


def available():
    return os.path.isdir(os.path.join(REF_ROOT, "src", "libhotspin"))


def build():
    sys.path.insert(0, ROOT)
    from tests.emu import build as emu
    src = os.path.join(REF_ROOT, "src", "libhotspin")
    gen = os.path.join(OUT, "emu_obj")
    os.makedirs(gen, exist_ok=True)
    inputs = [os.path.join(src, f) for f in os.listdir(src)] + [os.path.join(emu.HERE, f) for f in os.listdir(emu.HERE)]
    newest = max(os.path.getmtime(f) for f in inputs if os.path.isfile(f))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    # the reference's sources keep default visibility (not all of its exports are marked); the
    # emulated runtime stays hidden, private to this library
    flags = ["-std=c++17", "-O1", "-g", "-fPIC", "-Wno-unknown-pragmas", "-w", "-I" + emu.HERE, "-I" + src]
    jobs = []
    for f in sorted(os.listdir(src)):
        if f.endswith(".cu"):
            with open(os.path.join(src, f)) as fh:
                text = emu.rewrite(fh.read())
            dst = os.path.join(gen, f[:-3] + ".cpp")
            with open(dst, "w") as fh:
                fh.write("#line 1 \"%s\"\n" % os.path.join(src, f) + text)
            jobs.append((f, dst))
        elif f.endswith(".cpp"):
            jobs.append((f, os.path.join(src, f)))
    jobs.append(("emu_runtime.cpp", os.path.join(emu.HERE, "emu_runtime.cpp")))

    def compile_one(job):
        name, path = job
        obj = os.path.join(gen, os.path.splitext(name)[0] + ".o")
        extra = ["-fvisibility=hidden"] if name == "emu_runtime.cpp" else []
        p = subprocess.run(["g++"] + flags + extra + ["-c", path, "-o", obj], capture_output=True, text=True)
        return obj, (None if p.returncode == 0 else "%s:\n%s" % (name, p.stderr[-4000:]))
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        res = list(ex.map(compile_one, jobs))
    errs = [e for _, e in res if e]
    if errs:
        raise RuntimeError("emulation build of the reference library failed:\n" + "\n".join(errs))
    tmp = LIB + ".tmp%d" % os.getpid()
    p = subprocess.run(["g++", "-shared", "-o", tmp] + [o for o, _ in res], capture_output=True, text=True)
    if p.returncode:
        raise RuntimeError("emulation link of the reference library failed:\n" + p.stderr[-4000:])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build())
