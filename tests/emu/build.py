"""Build the library's CUDA sources for the CPU emulation of CUDA -- TEST INFRASTRUCTURE ONLY.

Each hotspin_b200/csrc/*.cu is copied with two textual rewrites a host compiler needs and
compiled as C++ against tests/emu/cuda_runtime.h (in place of the CUDA toolkit's headers):

* a launch ``kernel<<<grid, block, smem, stream>>>(args)`` becomes
  ``hsbemu::launch(kernel, grid, block, smem, stream)(args)``, which converts the arguments to
  the kernel's parameter types at the call, as a launch does, and runs the grid (or records it
  while the stream is being captured);
* ``extern __shared__ T name[];`` becomes a pointer to the launch's dynamic shared memory.

Everything else -- kernels, device functions, host code, the C ABI -- is the product's source
unchanged.  The result, libhsb200_emu.so, exports the same C ABI as the nvcc build; tests load
it explicitly (the product's loader never does).

    python tests/emu/build.py [--asan]
"""
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
SRC = os.path.join(ROOT, "hotspin_b200", "csrc")
OUT = os.path.join(HERE, "_build")

_SHARED = re.compile(r"extern\s+__shared__\s+(?:__align__\(\d+\)\s+)?([A-Za-z_][\w\s]*?)\s+(\w+)\s*\[\s*\]\s*;")


def _callee_start(s, i):
    """Start of the callee expression that ends just before position i (identifiers joined by
    ->, . or ::, each optionally followed by template arguments)."""
    j = i - 1
    while j >= 0 and s[j] in " \t":        # `kernel <<<...>>>`
        j -= 1
    while True:
        if j >= 0 and s[j] == ">":          # template arguments
            depth = 0
            while j >= 0:
                if s[j] == ">":
                    depth += 1
                elif s[j] == "<":
                    depth -= 1
                    if depth == 0:
                        break
                j -= 1
            j -= 1
        k = j
        while k >= 0 and (s[k].isalnum() or s[k] == "_"):
            k -= 1
        if k == j:
            raise ValueError("no callee before <<< at %d" % i)
        j = k
        if j >= 1 and s[j - 1:j + 1] == "->":
            j -= 2
        elif j >= 0 and s[j] == ".":
            j -= 1
        elif j >= 1 and s[j - 1:j + 1] == "::":
            j -= 2
        else:
            return j + 1


def rewrite(text):
    text = _SHARED.sub(lambda m: "%s* %s = (%s*)hsbemu::dyn_smem();" % (m.group(1), m.group(2), m.group(1)), text)
    out = []
    pos = 0
    while True:
        i = text.find("<<<", pos)
        if i < 0:
            out.append(text[pos:])
            break
        e = text.find(">>>", i)
        start = _callee_start(text, i)
        out.append(text[pos:start])
        out.append("hsbemu::launch(%s, %s)" % (text[start:i], text[i + 3:e]))
        pos = e + 3
    return "".join(out)


def _newest_input():
    files = [os.path.join(SRC, f) for f in os.listdir(SRC)] + [os.path.join(HERE, f) for f in os.listdir(HERE)]
    files += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    return max(os.path.getmtime(f) for f in files if os.path.isfile(f))


def build(asan=False, verbose=False):
    """Build (or reuse, when nothing it is made from changed) the emulation library."""
    os.makedirs(OUT, exist_ok=True)
    tag = "_asan" if asan else ""
    lib = os.path.join(OUT, "libhsb200_emu%s.so" % tag)
    if os.path.exists(lib) and os.path.getmtime(lib) >= _newest_input():
        return lib
    gen = os.path.join(OUT, "src" + tag)
    os.makedirs(gen, exist_ok=True)
    flags = ["-std=c++17", "-O1", "-g", "-fPIC", "-fvisibility=hidden", "-Wno-unknown-pragmas",
             "-I" + HERE, "-I" + SRC, "-I" + os.path.join(ROOT, "include")]
    if asan:
        flags += ["-fsanitize=address", "-fno-omit-frame-pointer"]
    jobs = []
    for f in sorted(os.listdir(SRC)):
        if not f.endswith(".cu"):
            continue
        dst = os.path.join(gen, f[:-3] + ".cpp")
        with open(os.path.join(SRC, f)) as fh:
            text = rewrite(fh.read())
        with open(dst, "w") as fh:
            fh.write("#line 1 \"%s\"\n" % os.path.join(SRC, f) + text)
        jobs.append((f, dst, os.path.join(gen, f[:-3] + ".o")))
    jobs.append(("emu_runtime.cpp", os.path.join(HERE, "emu_runtime.cpp"), os.path.join(gen, "emu_runtime.o")))

    def compile_one(job):
        name, src, obj = job
        cmd = ["g++"] + flags + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        p = subprocess.run(cmd, capture_output=True, text=True)
        return None if p.returncode == 0 else "emulation build of %s failed:\n%s" % (name, p.stderr[-6000:])
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        errs = [e for e in ex.map(compile_one, jobs) if e]
    if errs:
        raise RuntimeError("\n".join(errs))
    objs = [j[2] for j in jobs[:-1]]
    rt = jobs[-1][2]
    tmp = lib + ".tmp%d" % os.getpid()
    cmd = ["g++", "-shared", "-o", tmp] + objs + [rt] + (["-fsanitize=address"] if asan else [])
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode:
        raise RuntimeError("emulation link failed:\n" + p.stderr[-6000:])
    os.replace(tmp, lib)      # processes already holding the old file keep it
    return lib


if __name__ == "__main__":
    print(build(asan="--asan" in sys.argv, verbose="-v" in sys.argv))
