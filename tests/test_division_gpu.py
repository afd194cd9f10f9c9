"""The element maps take several quotients with a common divisor (1 + pz, the drift's p_s, the
bend's p_t, beta0, 6) from one rounded reciprocal and an FMA correction (Markstein's theorem).
The quotient must be the same bits as the division it replaces: checked on the device against
the device's own a / b on 4e9 pseudo-random pairs, a quarter of them next to rounding ties, and
through the tracking itself (the CPU host build of the same maps is bit-exact against the oracle,
which divides, in tests/test_hostcheck_cpu.py)."""
import importlib

import pytest

pytestmark = pytest.mark.gpu
lib = importlib.import_module("bmad-ecosystem_b200.lib")


def test_shared_reciprocal_division_is_exact():
    ctx = lib.Context(0)
    for seed in (1, 2, 3, 4):
        assert lib.selftest_division(ctx, 1_000_000_000, seed) == 0
    ctx.close()
