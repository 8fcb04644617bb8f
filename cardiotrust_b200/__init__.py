"""B200-native estimation epoch of CardioTrust (``run_epoch``).

The compute path is ``libcardiotrust_cuda.so`` (sm_100a kernels behind the C
ABI in ``include/cardiotrust_cuda.h``); this package holds its ctypes binding,
the reference-shaped host API (:mod:`.algorithm`) and the seeded scenario
generator (:mod:`.scenario`).
"""

__all__ = ["algorithm", "scenario", "build"]
