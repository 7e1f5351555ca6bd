"""B200-native pulse-profile engine (drop-in for the fizban007/gpu_ppm hot path).

The compute path is libppm_b200.so (hand-written sm_100a CUDA behind the C ABI
in include/ppm.h); this package is the thin Python host layer over it.
"""
from . import _abi  # noqa: F401
