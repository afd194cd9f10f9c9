"""Markstein's correction on the host (no GPU): RN(q + (a - b q) y) with q = RN(a y) and
y = RN(1/b) equals RN(a / b) -- the theorem the device maps' shared-reciprocal quotients rest
on -- checked with exact rational arithmetic for the FMA on random and tie-adjacent pairs."""
import math
import random
from fractions import Fraction as F


def fma(x, y, z):
    return float(F(x) * F(y) + F(z))


def div_rcp(a, b, y):
    q = a * y
    r = fma(-b, q, a)
    return fma(r, y, q)


def test_markstein_correction_matches_division():
    rng = random.Random(7)

    def rnd(lo=-60, hi=60):
        return rng.choice((-1, 1)) * (1 + rng.getrandbits(52) / 2 ** 52) * 2.0 ** rng.randint(lo, hi)

    cases = [(rnd(), rnd()) for _ in range(20000)]
    for _ in range(10000):
        b, q = rnd(-5, 5), rnd(-5, 5)
        p = b * q
        cases += [(p, b), (math.nextafter(p, math.inf), b), (math.nextafter(p, -math.inf), b)]
    special = [1.0, 1 + 2 ** -52, 2 - 2 ** -52, 1.5, 2 - 2 ** -26, 6.0]
    cases += [(s * ma * 2.0 ** e, mb) for ma in special for mb in special for e in range(-3, 4) for s in (1, -1)]
    for a, b in cases:
        assert div_rcp(a, b, 1.0 / b) == a / b, (a.hex(), b.hex())
