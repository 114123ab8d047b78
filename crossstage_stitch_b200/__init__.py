"""B200-native (sm_100a) implementation of CrossStage-Stitch's per-pair
registration chain: S2 FAST-9 + NMS, S3 ORB orientation + rBRIEF, S4
Hamming kNN-2 + ratio test, S5 MSAC 4-point homography.

The stages live in libstitch_b200.so (hand-written CUDA + C++ host code)
behind the reference's own stage API and a C ABI (include/stitch_b200.h);
this package is the ctypes binding plus the Python-side runners.
"""
from ._abi import LIB_PATH, Status, StageError, load  # noqa: F401

__all__ = ["LIB_PATH", "Status", "StageError", "load"]
