"""B200-native implementation of CFFC's 2D Euler finite-volume path.

The compute path is hand-written sm_100a CUDA in ``libcffc_e2d.so`` (sources
in ``csrc/``), reached through the C ABI of ``include/cffc_e2d.h``.
"""
from . import cases  # noqa: F401
