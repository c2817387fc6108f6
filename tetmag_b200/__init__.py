"""tetmag_b200: B200-native effective-field + LLG right-hand side of tetmag.

The compute path is libtmb.so (hand-written sm_100a CUDA behind a C ABI,
include/tmb.h); this package is its host-side binding and workload harness.
"""
from ._lib import LIB_PATH, TmbError, lib  # noqa: F401

__all__ = ["LIB_PATH", "TmbError", "lib"]
