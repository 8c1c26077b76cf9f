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
