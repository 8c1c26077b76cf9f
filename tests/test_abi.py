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
