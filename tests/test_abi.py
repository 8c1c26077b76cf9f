"""The C-ABI library loads and exports every symbol its headers declare (no GPU needed)."""
import ctypes
import subprocess

from hotspin_b200 import _lib


def test_library_builds_and_loads():
    from hotspin_b200 import build
    build.build()
    lib = _lib.load()
    assert lib.hsb_version() >= 1


def test_every_declared_symbol_is_exported():
    lib = _lib.load()
    names = _lib.exported_symbols_from_headers()
    assert len(names) > 50
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert names <= exported, sorted(names - exported)


def test_python_signatures_match_the_header_prototypes():
    """Every ctypes signature the bindings set (hotspin_b200/_lib.py) has the header
    prototype's parameter count, and each parameter and result the C type's width and kind."""
    import os
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = "".join(open(os.path.join(root, "include", f)).read() for f in sorted(os.listdir(os.path.join(root, "include"))))
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    handles = ("hsb_sim", "hsb_batch", "hsb_demag_plan", "hsb_fft_plan")

    def ctype_of(decl):
        d = re.sub(r"\bconst\b", "", decl).strip()
        d = re.sub(r"\s+\w+$", "", d) if not d.endswith("*") else d   # drop the parameter name
        d = d.replace(" ", "")
        if d in handles or d == "void*":
            return ctypes.c_void_p
        if d.endswith("*"):
            base = d[:-1]
            if base == "char":
                return ctypes.c_char_p
            if base in handles:
                return ctypes.POINTER(ctypes.c_void_p)
            return ctypes.POINTER(ctype_of(base + " x"))
        return {"int": ctypes.c_int, "int32_t": ctypes.c_int32, "int64_t": ctypes.c_int64, "long": ctypes.c_long,
                "double": ctypes.c_double, "float": ctypes.c_float, "uint64_t": ctypes.c_uint64,
                "hsb_sim_desc": _lib.SimDesc}[d]

    def same(a, b):
        if a is None or b is None:
            return a is b
        if b is ctypes.c_void_p and (a is ctypes.c_void_p or a.__name__.startswith("LP_")):
            return True       # device addresses and opaque buffers are bound as void*
        if hasattr(a, "_type_") and hasattr(b, "_type_") and a.__name__.startswith("LP_"):
            return b.__name__.startswith("LP_") and same(a._type_, b._type_)
        return ctypes.sizeof(a) == ctypes.sizeof(b) and a._type_ == b._type_ if hasattr(a, "_type_") and \
            isinstance(a._type_, str) and hasattr(b, "_type_") and isinstance(b._type_, str) else a is b

    bad = []
    for name, (res, args) in _lib._SIGS.items():
        m = re.search(r"([\w\s\*]+?)\b" + name + r"\s*\(([^)]*)\)\s*;", src)
        assert m, "no prototype for " + name
        params = [p.strip() for p in m.group(2).split(",") if p.strip() and p.strip() != "void"]
        ret = m.group(1).strip().split("\n")[-1].strip()
        want_res = None if ret == "void" else ctype_of(ret + (" x" if not ret.endswith("*") else ""))
        if len(params) != len(args):
            bad.append((name, "parameter count", len(params), len(args)))
            continue
        if not same(want_res, res):
            bad.append((name, "result", ret, res))
        for p, a in zip(params, args):
            if not same(ctype_of(p), a):
                bad.append((name, p, a))
    assert not bad, bad


def test_errors_are_reported_not_aborted():
    lib = _lib.load()
    h = ctypes.c_void_p()
    d = _lib.SimDesc()          # all zero: invalid
    rc = lib.hsb_sim_create(ctypes.byref(d), ctypes.byref(h))
    assert rc == 1 and b"bad size" in lib.hsb_last_error()
    assert lib.hsb_sim_step(None, 1) == 1


def test_descriptor_layout_agrees_in_c_python_and_the_library(tmp_path):
    """A C program compiled against include/hotspin_b200.h and linked to the library sees the
    same hsb_sim_desc layout as the Python mirror and as the library itself, and calls it."""
    import os
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    src = tmp_path / "abi.c"
    src.write_text(r'''
#include <stddef.h>
#include <stdio.h>
#include "hotspin_b200.h"
int main(void) {
    printf("%zu %zu %zu %zu %zu %d %d %llu\n", sizeof(hsb_sim_desc), offsetof(hsb_sim_desc, seed),
           offsetof(hsb_sim_desc, maxdt), offsetof(hsb_sim_desc, laser_table),
           offsetof(hsb_sim_desc, laser_npts), hsb_sim_desc_bytes(), hsb_version(),
           (unsigned long long)hsb_crc64_iso("123456789", 9));
    return 0;
}
''')
    exe = tmp_path / "abi"
    libdir = os.path.dirname(_lib.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-I", inc, str(src), "-L", libdir, "-lhsb200", "-Wl,-rpath," + libdir,
                    "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    size, seed, maxdt, tab, npts, lib_size, version, crc = (int(x) for x in out)
    D = _lib.SimDesc
    assert size == ctypes.sizeof(D) == lib_size == _lib.load().hsb_sim_desc_bytes()
    assert (seed, maxdt, tab, npts) == (D.seed.offset, D.maxdt.offset, D.laser_table.offset, D.laser_npts.offset)
    assert version >= 1
    assert crc == 0xB90956C775A41001      # CRC-64/GO-ISO check value of "123456789"


def test_every_descriptor_field_at_the_same_offset(tmp_path):
    """Every field of hsb_sim_desc sits at the same offset in the public header, in the Python
    mirror and in the library's own copy of the struct (hsb_desc.h, compiled here as host C++)."""
    import os
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    names = [f[0] for f in _lib.SimDesc._fields_]
    body = open(os.path.join(root, "hotspin_b200", "csrc", "hsb_desc.h")).read()
    mirror = re.search(r"struct hsb_sim_desc \{.*?\n\};", body, re.S).group(0)
    prints = "".join('    printf("%%s %%zu %%zu\\n", "%s", offsetof(hsb_sim_desc, %s), offsetof(lib::hsb_sim_desc, %s));\n'
                     % (n, n, n) for n in names)
    src = tmp_path / "layout.cpp"
    src.write_text("#include <stddef.h>\n#include <stdint.h>\n#include <stdio.h>\n#include \"hotspin_b200.h\"\n"
                   "namespace lib {\n" + mirror + "\n}\nint main() {\n" + prints +
                   '    printf("sizeof %zu %zu\\n", sizeof(hsb_sim_desc), sizeof(lib::hsb_sim_desc));\n    return 0;\n}\n')
    exe = tmp_path / "layout"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines()
    rows = {l.split()[0]: tuple(int(x) for x in l.split()[1:]) for l in out}
    D = _lib.SimDesc
    assert rows["sizeof"] == (ctypes.sizeof(D), ctypes.sizeof(D))
    bad = [(n, rows[n], getattr(D, n).offset) for n in names if rows[n] != (getattr(D, n).offset,) * 2]
    assert not bad, bad
    # and no field of the header is missing from the Python mirror
    hdr = open(os.path.join(root, "include", "hotspin_b200.h")).read()
    pub = re.search(r"typedef struct hsb_sim_desc \{(.*?)\n\} hsb_sim_desc;", hdr, re.S)
    if pub:
        decl = re.sub(r"/\*.*?\*/|//[^\n]*", "", pub.group(1), flags=re.S)
        fields = set(re.findall(r"(\w+)\s*(?:\[\d+\])?\s*[;,]", decl))
        assert fields <= set(names), sorted(fields - set(names))


def _desc(**kw):
    from hotspin_b200.sim import make_desc
    base = dict(size=(1, 8, 8), cellsize=(1e-9,) * 3, msat0T0=8e5, lex=5e-9, solver="rk4", dt=1e-14)
    base.update(kw)
    return make_desc(**base)


def _create(d):
    lib = _lib.load()
    h = ctypes.c_void_p()
    return lib.hsb_sim_create(ctypes.byref(d), ctypes.byref(h)), lib.hsb_last_error()


def test_limits_are_checked_before_any_device_work():
    """Argument checks run on the host before the first CUDA call (so they also hold here):
    grids above 2^28 cells, bad laser tables, solver/tolerance errors, and demag plans whose
    padded lengths are not powers of two."""
    rc, msg = _create(_desc(size=(1024, 1024, 512)))
    assert rc == 4 and b"2^28" in msg
    rc, msg = _create(_desc(ttm=True, gamma_e=700.0, c_l=3e6, laser_p0=1e20,
                            laser_table=[(0.0, 0.0), (1e-13, 1.0), (1e-13, 0.5)]))
    assert rc == 1 and b"not increasing" in msg
    rc, msg = _create(_desc(ttm=True, gamma_e=700.0, c_l=3e6, laser_table=[(0.0, 1.0)]))
    assert rc == 1 and b"laser_npts" in msg
    rc, msg = _create(_desc(solver="dp45", rtol=0.0))
    assert rc == 1 and b"rtol" in msg
    rc, msg = _create(_desc(llb=True, tc=0.0))
    assert rc == 1 and b"llb" in msg
    lib = _lib.load()
    plan = ctypes.c_void_p()
    # an open axis whose padding is not a power of two runs embedded in a larger grid; a
    # periodic one cannot (its transform length is the grid's own) and is refused
    size = (ctypes.c_int * 3)(3, 8, 8)
    cs = (ctypes.c_double * 3)(1e-9, 1e-9, 1e-9)
    pbc = (ctypes.c_int * 3)(1, 0, 0)
    assert lib.hsb_demag_plan_create(size, cs, pbc, 6, None, ctypes.byref(plan)) == 4
    assert b"power of two" in lib.hsb_last_error()


def test_batches_refuse_what_they_do_not_support():
    lib = _lib.load()
    nbytes = ctypes.c_int64()
    d = _desc(size=(1, 8, 10), solver="dp45")            # a2 not a multiple of 4
    assert lib.hsb_batch_footprint(ctypes.byref(d), 4, ctypes.byref(nbytes)) == 4
    d = _desc(size=(1, 8, 8), solver="dp45", ttm=True, gamma_e=700.0, c_l=3e6, laser_p0=1e20,
              laser_table=[(0.0, 0.0), (1e-13, 1.0)])
    assert lib.hsb_batch_footprint(ctypes.byref(d), 4, ctypes.byref(nbytes)) == 4
    assert b"batches" in lib.hsb_last_error()
    d = _desc(size=(1, 8, 8), solver="dp45")
    assert lib.hsb_batch_footprint(ctypes.byref(d), 0, ctypes.byref(nbytes)) == 1
    d = _desc(size=(1, 12, 8), solver="dp45", demag=True)  # demag classes: powers of two only
    assert lib.hsb_batch_footprint(ctypes.byref(d), 4, ctypes.byref(nbytes)) == 4
    assert b"powers of two" in lib.hsb_last_error()


def test_dropins_export_every_name_the_go_sequence_replay_binds():
    """oracle/replay.py binds these reference names through ctypes; libhsb200.so must export
    each of them so the replay (and a Go build linking the drop-ins) can run on it."""
    import ctypes

    from hotspin_b200 import _lib
    from oracle import replay
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in replay._SIGS if not hasattr(lib, n)]
    assert not missing, missing
