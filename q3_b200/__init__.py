"""q3_b200 -- B200-native plane-wave H|psi> and block-Davidson (sm_100a).

The compute lives in ``libq3b.so`` (hand-written CUDA for sm_100a behind the C
ABI of ``include/q3b.h``); this package is its host-side mirror of the
reference's operator interfaces plus the seeded synthetic inputs.
"""
from ._lib import FP64, MIXED, Q3BError  # noqa: F401

__all__ = ["FP64", "MIXED", "Q3BError"]
