"""Reader/writer of hotspin's ``#dump002`` frame format (test infrastructure).

Layout (src/hotspin-core/dump/writer.go:46-76, reader.go:29-70): 8-byte magic, u64 number
of components, 3 x u64 mesh size (program order), 3 x f64 cell size, 8-byte unit string,
f64 time, 8-byte time unit, 8-byte label, 8-byte data unit, u64 precision (4), float32
payload ``[c][i][j][k]``, u64 CRC-64 (ISO polynomial, Go's ``hash/crc64`` convention,
computed over every preceding byte of the frame; 0 means "not set").
"""
import struct

import numpy as np

MAGIC = b"#dump002"
_POLY = 0xD800000000000000  # ISO polynomial, reflected


def _table():
    t = np.zeros(256, dtype=np.uint64)
    for i in range(256):
        c = i
        for _ in range(8):
            c = (c >> 1) ^ _POLY if c & 1 else c >> 1
        t[i] = c
    return [int(x) for x in t]


_TABLE = _table()


def crc64_iso(data: bytes) -> int:
    """CRC-64/ISO as in Go's hash/crc64 (init and final xor all-ones, reflected)."""
    crc = 0xFFFFFFFFFFFFFFFF
    tab = _TABLE
    for b in data:
        crc = tab[(crc ^ b) & 0xFF] ^ (crc >> 8)
    return crc ^ 0xFFFFFFFFFFFFFFFF


def _str8(s):
    b = s.encode() if isinstance(s, str) else bytes(s)
    return (b + b"\0" * 8)[:8]


def read_dump(path, check_crc=True):
    """Return (data float64 array (ncomp, n0, n1, n2), header dict)."""
    raw = open(path, "rb").read()
    if raw[:8] != MAGIC:
        raise ValueError("dump: bad magic number: %r" % raw[:8])
    ncomp = struct.unpack("<Q", raw[8:16])[0]
    mesh = struct.unpack("<3Q", raw[16:40])
    step = struct.unpack("<3d", raw[40:64])
    munit = raw[64:72]
    t = struct.unpack("<d", raw[72:80])[0]
    tunit, label, dunit = raw[80:88], raw[88:96], raw[96:104]
    prec = struct.unpack("<Q", raw[104:112])[0]
    n = ncomp * mesh[0] * mesh[1] * mesh[2]
    end = 112 + 4 * n
    data = np.frombuffer(raw[112:end], dtype="<f4").reshape((ncomp,) + tuple(mesh))
    crc = struct.unpack("<Q", raw[end:end + 8])[0]
    if check_crc and crc != 0:
        mine = crc64_iso(raw[:end])
        if mine != crc:
            raise ValueError("dump CRC error: expected %016x, got %016x" % (crc, mine))
    hdr = dict(ncomp=ncomp, mesh=mesh, cellsize=step, meshunit=munit, time=t, timeunit=tunit,
               label=label, dataunit=dunit, precision=prec, crc=crc)
    return data.astype(np.float64), hdr


def write_dump(path, data, cellsize=(1.0, 1.0, 1.0), time=0.0, label="", unit="",
               crc=True):
    data = np.asarray(data, dtype="<f4")
    if data.ndim == 3:
        data = data[None]
    body = bytearray()
    body += MAGIC
    body += struct.pack("<Q", data.shape[0])
    body += struct.pack("<3Q", *data.shape[1:])
    body += struct.pack("<3d", *cellsize)
    body += _str8("m")
    body += struct.pack("<d", time)
    body += _str8("s")
    body += _str8(label)
    body += _str8(unit)
    body += struct.pack("<Q", 4)
    body += data.tobytes()
    body += struct.pack("<Q", crc64_iso(bytes(body)) if crc else 0)
    with open(path, "wb") as f:
        f.write(bytes(body))
