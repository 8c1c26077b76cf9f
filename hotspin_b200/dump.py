"""hotspin's ``#dump002`` frame files: write a simulation's fields, read them back.

A frame (dump/writer.go:46-76, dump/reader.go:29-70) is: the 8-byte magic ``#dump002``; u64
component count; 3 x u64 mesh size in program order (z, y, x); 3 x f64 cell size; an 8-byte
mesh unit; f64 time; an 8-byte time unit; an 8-byte label; an 8-byte data unit; u64 precision
(4 = float32); the float32 payload ``[component][z][y][x]`` (component 0 = user z); and a u64
CRC-64/ISO over every preceding byte of the frame (0 = not set).  A file may hold several
frames back to back.  The CRC runs in the native library (``hsb_crc64_iso``).
"""
import ctypes
import struct

import numpy as np

from . import _lib

MAGIC = b"#dump002"
_HEADER = struct.Struct("<8sQ3Q3d8sd8s8s8sQ")


def _text8(s):
    b = s.encode() if isinstance(s, str) else bytes(s)
    if len(b) > 8:
        raise ValueError("dump: unit and label strings hold at most 8 bytes, got %r" % b)
    return b.ljust(8, b"\0")


def crc64(data) -> int:
    """CRC-64/ISO of a bytes-like object, as the dump writer seals frames."""
    a = np.frombuffer(data, dtype=np.uint8)
    if a.size == 0:
        return 0
    return int(_lib.load().hsb_crc64_iso(ctypes.c_void_p(a.ctypes.data), a.size))


def frame_bytes(data, cellsize, time=0.0, label="", unit="", mesh_unit="m", time_unit="s", crc=True) -> bytes:
    """One frame of `data` (ncomp, n0, n1, n2) or (n0, n1, n2), stored as float32."""
    a = np.ascontiguousarray(data, dtype="<f4")
    if a.ndim == 3:
        a = a[None]
    if a.ndim != 4:
        raise ValueError("dump: data must be (ncomp, n0, n1, n2), got shape %s" % (a.shape,))
    head = _HEADER.pack(MAGIC, a.shape[0], *a.shape[1:], *[float(c) for c in cellsize], _text8(mesh_unit),
                        float(time), _text8(time_unit), _text8(label), _text8(unit), 4)
    body = head + a.tobytes()
    return body + struct.pack("<Q", crc64(body) if crc else 0)


def write(path, data, cellsize, time=0.0, label="", unit="", append=False, crc=True):
    """Write (or append) one frame to `path`."""
    with open(path, "ab" if append else "wb") as f:
        f.write(frame_bytes(data, cellsize, time, label, unit, crc=crc))


def write_simulation(path, sim, name="m", cellsize=None, append=False):
    """Frame of a Simulation's field `name` (its FP32 state as FP64 through hsb_sim_get) at
    the handle's current time."""
    data = sim.get(name)
    t = sim.status()["t"]
    cs = cellsize if cellsize is not None else tuple(sim.desc.cellsize)
    write(path, data, cs, time=t, label=name, append=append)


def read(path, check_crc=True):
    """All frames of `path`: a list of (float32 array (ncomp, n0, n1, n2), header dict)."""
    raw = open(path, "rb").read()
    frames, pos = [], 0
    while pos < len(raw):
        if len(raw) - pos < _HEADER.size:
            raise ValueError("dump: truncated header at byte %d" % pos)
        (magic, ncomp, n0, n1, n2, c0, c1, c2, munit, t, tunit, label, dunit,
         prec) = _HEADER.unpack_from(raw, pos)
        if magic != MAGIC:
            raise ValueError("dump: bad magic %r at byte %d" % (magic, pos))
        if prec != 4:
            raise ValueError("dump: precision %d is not supported (float32 frames only)" % prec)
        n = ncomp * n0 * n1 * n2
        end = pos + _HEADER.size + 4 * n
        if end + 8 > len(raw):
            raise ValueError("dump: truncated payload at byte %d" % pos)
        data = np.frombuffer(raw, dtype="<f4", count=n, offset=pos + _HEADER.size).reshape(ncomp, n0, n1, n2)
        stored = struct.unpack_from("<Q", raw, end)[0]
        if check_crc and stored != 0:
            got = crc64(raw[pos:end])
            if got != stored:
                raise ValueError("dump: CRC mismatch in the frame at byte %d: stored %016x, computed %016x"
                                 % (pos, stored, got))
        frames.append((data.copy(), dict(ncomp=ncomp, mesh=(n0, n1, n2), cellsize=(c0, c1, c2),
                                         mesh_unit=munit.rstrip(b"\0").decode(errors="replace"), time=t,
                                         time_unit=tunit.rstrip(b"\0").decode(errors="replace"),
                                         label=label.rstrip(b"\0").decode(errors="replace"),
                                         unit=dunit.rstrip(b"\0").decode(errors="replace"), crc=stored)))
        pos = end + 8
    return frames
