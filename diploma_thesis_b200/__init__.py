"""B200-native (sm_100a) implementation of AR_Sim's per-step rigid-body pipeline.

The compute path is ``libarsim.so`` (CUDA, built in-tree by ``diploma_thesis_b200.build``)
behind the C ABI in ``include/arsim.h``.  This package holds the Python host interface
(``api``), the ctypes binding (``_lib``), scene generators (``scenes``), the autotuner
(``autotune``) and the continuous-batching server (``serve``).  Importing ``api`` requires
the built library; nothing falls back to the CPU.
"""
__all__ = ["api", "scenes"]
