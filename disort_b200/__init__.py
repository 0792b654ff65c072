"""disort_b200 — B200-native DISORT spectral engine (FP64, sm_100a).

The C ABI lives in include/dsp.h (libdsp.so under disort_b200/lib); ``capi``
is its ctypes mirror.
"""
from . import capi  # noqa: F401

__version__ = "0.1.0"
