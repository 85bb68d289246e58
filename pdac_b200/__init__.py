"""B200-native (sm_100a) engine for PDAC's per-time-step hot path.

The compute path is the CUDA library ``pdac_b200/_lib/libpdac_b200.so``
behind the C ABI of ``include/pdac_gpu.h``; :mod:`pdac_b200.engine` binds it
with ctypes.  :mod:`pdac_b200.deck` and :mod:`pdac_b200.setup_state` are the
host-side input reader and run set-up.
"""
__version__ = "0.1.0"
