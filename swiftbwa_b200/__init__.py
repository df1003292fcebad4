"""swiftbwa_b200 -- B200-native (sm_100a) Smith-Waterman hot path of swiftbwa.

The product is libswb_cuda.so (C ABI in include/swb_cuda.h); this package
holds its sources (csrc/), the build recipe (build.py), the ctypes binding
(abi.py) and a host mirror of the reference's Alignment API (alignment.py).
"""
from .abi import Scoring, load_library  # noqa: F401
