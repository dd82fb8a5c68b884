"""CoolBubble's lattice-evolution path on the B200 (sm_100a).

The compute lives in the CUDA library ``lib/libcoolbubble_b200.so`` (C ABI in
include/coolbubble_b200.h); this package is its Python binding and a mirror
of the reference's Bubble interface for scripting and tests.
"""
from ._lib import CBError, CB_FP32C, CB_FP64  # noqa: F401  (raises if the library is not built)
from .bubble import Bubble, make_params  # noqa: F401

__all__ = ["Bubble", "make_params", "CBError", "CB_FP64", "CB_FP32C"]
