"""pentago_b200: B200-native (sm_100a) kernels for pentago's backward solve.

The compute lives in the CUDA library pentago_b200/_lib/libpentago_b200.so
(C ABI: include/pentago_b200.h); this package is the Python mirror of the
reference's interfaces for the hot path.
"""
from . import capi  # noqa: F401
