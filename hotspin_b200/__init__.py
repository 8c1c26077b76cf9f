"""hotspin_b200: B200-native (sm_100a) implementation of hotspin's solver hot path.

The compute lives in libhsb200.so (hotspin_b200/csrc, built by ``python -m
hotspin_b200.build``); this package holds the ctypes binding (``_lib``), the simulation
handle wrapper (``sim``) and the script-level mirror of hotspin's Python client (``api``).
"""
from . import _lib  # noqa: F401

__all__ = ["_lib"]
