"""B200-native (sm_100a, FP64) replacement for Bmad's multi-particle bmad_standard tracking path."""
from . import abi  # noqa: F401
