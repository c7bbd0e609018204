"""B200-native implementation of the DNS_GKM_LPT hot path.

The product is libgkm_b200.so (CUDA sm_100a kernels behind the C ABI of
include/gkm.h); this package holds its sources (csrc/), the build step
(build.py), the ctypes binding (_capi.py), a host mirror of the reference's
interface (solver.py) and the seeded initial-condition generator (ic.py).
"""
from .ic import Params  # noqa: F401

__all__ = ["Params"]
