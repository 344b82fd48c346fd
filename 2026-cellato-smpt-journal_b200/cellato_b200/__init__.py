"""Python mirror of the B200 bit-plane hot path (C ABI in include/cellato_b200.h).

``lib``     ctypes binding of the shared library (no fallback: it must be built)
``inputs``  seeded synthetic initial grids
``device``  device-resident planes in torch CUDA memory
"""
from . import inputs, lib  # noqa: F401

__all__ = ["inputs", "lib"]
