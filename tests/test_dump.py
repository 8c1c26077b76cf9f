"""hotspin_b200.dump against the oracle's #dump002 reader / writer and the reference's own
dump files (when the reference checkout is present)."""
import glob
import os

import numpy as np
import pytest

from hotspin_b200 import dump
from oracle import REF_ROOT
from oracle import dump as odump


def test_crc_matches_the_oracle():
    rng = np.random.default_rng(0)
    for n in (0, 1, 7, 64, 1000):
        b = rng.integers(0, 256, size=n, dtype=np.uint8).tobytes()
        assert dump.crc64(b) == (odump.crc64_iso(b) if n else 0)


def test_frames_round_trip_through_both_implementations(tmp_path):
    rng = np.random.default_rng(1)
    a = rng.normal(size=(3, 2, 5, 7)).astype(np.float32)
    b = rng.normal(size=(1, 2, 5, 7)).astype(np.float32)
    p = str(tmp_path / "x.dump")
    dump.write(p, a, (3e-9, 2e-9, 1e-9), time=1.5e-12, label="m")
    data, hdr = odump.read_dump(p)                     # the oracle reader checks the CRC
    assert np.array_equal(data, a.astype(np.float64))
    assert hdr["mesh"] == (2, 5, 7) and hdr["cellsize"] == (3e-9, 2e-9, 1e-9) and hdr["time"] == 1.5e-12
    dump.write(p, b, (3e-9, 2e-9, 1e-9), time=2e-12, label="Te", append=True)
    frames = dump.read(p)
    assert len(frames) == 2
    assert np.array_equal(frames[0][0], a) and np.array_equal(frames[1][0], b)
    assert frames[1][1]["label"] == "Te" and frames[1][1]["time"] == 2e-12
    q = str(tmp_path / "y.dump")
    odump.write_dump(q, a, cellsize=(1.0, 2.0, 3.0), time=3.0, label="m")
    (got, h), = dump.read(q)
    assert np.array_equal(got, a) and h["cellsize"] == (1.0, 2.0, 3.0)


def test_corrupted_frame_is_refused(tmp_path):
    p = str(tmp_path / "z.dump")
    dump.write(p, np.ones((3, 1, 2, 2), np.float32), (1.0, 1.0, 1.0))
    raw = bytearray(open(p, "rb").read())
    raw[120] ^= 0x01
    open(p, "wb").write(bytes(raw))
    with pytest.raises(ValueError, match="CRC"):
        dump.read(p)


REF_DUMPS = sorted(glob.glob(os.path.join(REF_ROOT, "tests", "*", "*.dump")))


@pytest.mark.skipif(not REF_DUMPS, reason="the reference checkout is not present")
def test_reads_the_reference_dump_files():
    for path in REF_DUMPS:
        frames = dump.read(path)
        want, hdr = odump.read_dump(path)
        assert len(frames) >= 1
        assert np.array_equal(frames[0][0].astype(np.float64), want)
        assert frames[0][1]["crc"] == hdr["crc"]
