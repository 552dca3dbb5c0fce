"""B200-native (sm_100a) meshless RBF-FD multigrid hot path.

The compute runs in libmgm.so (hand-written CUDA + C ABI, include/mgm.h);
this package holds the synthetic cloud generators, the ctypes binding and a
Python mirror of the reference's call surface.
"""
from . import clouds  # noqa: F401
from ._lib import (BC_LID, BC_TAYLOR_COUETTE, FIELD, GUESS_EXTRAPOLATE, GUESS_LEARNED, MODE_FP32_IR,  # noqa: F401
                   MODE_FP64, MODE_REFERENCE, MgmError, load)

__all__ = ["clouds", "load", "MgmError", "MODE_REFERENCE", "MODE_FP64", "MODE_FP32_IR", "BC_LID",
           "BC_TAYLOR_COUETTE", "FIELD", "GUESS_EXTRAPOLATE", "GUESS_LEARNED"]
