"""B200-native (sm_100a, FP64) replacement for Bmad's multi-particle bmad_standard tracking path.

Layers: ``abi`` (ctypes mirror of include/bmadgpu.h), ``lib`` (bindings of libbmadgpu.so, the
C-ABI drop-in), ``rings`` (synthetic benchmark rings and matched beams).
"""
from . import abi  # noqa: F401
