"""The correctly rounded transcendentals (csrc/crmath.cuh), host build, against mpmath.

Each function is evaluated on seeded arguments over the ranges the tracking maps use and far
beyond them (tiny, subnormal, near the reduction and series thresholds, huge arguments for the
Payne-Hanek reduction, the overflow edge of sinh/cosh), and on the special values of C99 Annex F.
The reference value is mpmath's at 200 bits (1300 for sin/cos beyond 2^20), rounded to nearest
even: every result must be that double, bit for bit. The device build of the same source is
checked against this host build on the GPU (tests/test_crmath_gpu.py)."""
import ctypes
import math
import os
import subprocess

import mpmath as mp
import numpy as np
import pytest

from conftest import ROOT

LIB = os.path.join(ROOT, "bmad-ecosystem_b200", "_build", "libbmadgpu_crmath.so")
FN = {"sin": 0, "cos": 1, "asin": 2, "atan2": 3, "sinh": 4, "cosh": 5, "exp": 8, "tan": 9}


@pytest.fixture(scope="module")
def cr():
    if not os.path.exists(LIB):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "bmad-ecosystem_b200", "csrc"), "hostcheck-lib"])
    lib = ctypes.CDLL(LIB)
    D = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    lib.bmadgpu_cr_eval_host.argtypes = [ctypes.c_int, D, D, D, ctypes.c_long]
    for f in (lib.bmadgpu_cr_sincos, lib.bmadgpu_cr_sinhcosh):
        f.argtypes = [ctypes.c_double, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    return lib


def evaluate(lib, name, a, b=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.zeros_like(a) if b is None else np.ascontiguousarray(b, dtype=np.float64)
    out = np.empty_like(a)
    lib.bmadgpu_cr_eval_host(FN[name], a, b, out, len(a))
    return out


def exact(name, a, b=0.0):
    """mpmath's value rounded to the nearest double (ties to even)."""
    if a == 0 and name in ("sin", "asin", "sinh"):
        return a                     # odd functions keep the sign of zero (mpmath has no -0)
    if a == 0 and name == "tan":
        return a
    prec = 1300 if name in ("sin", "cos", "tan") and abs(a) >= 2.0 ** 20 else 200
    with mp.workprec(prec):
        x = mp.mpf(a)
        if name == "sin":
            v = mp.sin(x)
        elif name == "cos":
            v = mp.cos(x)
        elif name == "asin":
            v = mp.asin(x)
        elif name == "atan2":
            v = mp.atan2(x, mp.mpf(b))
        elif name == "sinh":
            v = mp.sinh(x)
        elif name == "exp":
            v = mp.exp(x)
            if v < mp.mpf(2) ** -1022:   # subnormal range: round on the grid of 2^-1074
                q = v / mp.mpf(2) ** -1074
                n = mp.floor(q)
                n = n + 1 if (q - n > 0.5 or (q - n == 0.5 and int(n) % 2)) else n
                return float(n) * 2.0 ** -1074
        elif name == "tan":
            v = mp.tan(x)
        else:
            v = mp.cosh(x)
        if abs(v) > mp.mpf(2) ** 1024 * (1 - mp.mpf(2) ** -54):
            return math.copysign(math.inf, float(mp.sign(v)))
        return float(v)


def check(lib, name, a, b=None):
    got = evaluate(lib, name, a, b)
    bad = []
    for i in range(len(got)):
        want = exact(name, a[i], 0.0 if b is None else b[i])
        if not (got[i] == want and math.copysign(1, got[i]) == math.copysign(1, want)):
            bad.append((a[i], None if b is None else b[i], got[i], want))
    assert not bad, "%s: %d of %d not correctly rounded, e.g. %r" % (name, len(bad), len(got), bad[:3])


def logu(rng, lo, hi, n, signed=True):
    x = np.exp2(rng.uniform(lo, hi, n))
    return x * rng.choice([-1.0, 1.0], n) if signed else x


N = 1500


@pytest.mark.parametrize("name", ["sin", "cos"])
def test_sin_cos(cr, name):
    rng = np.random.default_rng(11)
    for a in (rng.uniform(-0.8, 0.8, N), rng.uniform(-4, 4, N), rng.uniform(-1e5, 1e5, N),
              logu(rng, -40, 20, N), logu(rng, 20, 1023, N // 3),
              # next to multiples of pi/2 (the cancellation of the reduction)
              np.array([k * math.pi / 2 * (1 + e) for k in range(1, 40) for e in (-3e-16, 0, 3e-16, 1e-12)])):
        check(cr, name, a)


def test_asin(cr):
    rng = np.random.default_rng(12)
    for a in (rng.uniform(-1, 1, N), logu(rng, -40, -1, N), 1 - logu(rng, -52, -2, N, signed=False),
              -(1 - logu(rng, -52, -2, N, signed=False)), rng.uniform(-1e-3, 1e-3, N)):
        check(cr, "asin", a)


def test_atan2(cr):
    rng = np.random.default_rng(13)
    y = np.concatenate([logu(rng, -30, 30, N), rng.uniform(-1, 1, N), logu(rng, -1000, 1000, N // 2),
                        rng.uniform(0.01, 0.05, N)])
    x = np.concatenate([logu(rng, -30, 30, N), rng.uniform(-1, 1, N), logu(rng, -1000, 1000, N // 2),
                        -rng.uniform(0.9, 1.1, N)])
    check(cr, "atan2", y, x)
    # |y| = |x| (the octant boundary) and neighbours
    v = logu(rng, -20, 20, 200, signed=False)
    for s in (1.0, 1 + 2.0 ** -52, 1 - 2.0 ** -53):
        check(cr, "atan2", v * s, v)
        check(cr, "atan2", -v * s, -v)


@pytest.mark.parametrize("name", ["sinh", "cosh"])
def test_sinh_cosh(cr, name):
    rng = np.random.default_rng(14)
    for a in (rng.uniform(-0.25, 0.25, N), rng.uniform(-3, 3, N), rng.uniform(-710.4, 710.4, N),
              logu(rng, -40, -2, N), rng.uniform(709.5, 710.6, N // 3),
              np.array([0.25, -0.25, 0.25 * (1 - 2.0 ** -53), 0.25 * (1 + 2.0 ** -52), 2.0 ** -26, 2.0 ** -27])):
        check(cr, name, a)


def test_special_values(cr):
    inf, nan = math.inf, math.nan
    tiny = 5e-324
    sv = [0.0, -0.0, tiny, -tiny, 2.2250738585072014e-308, 1.0, -1.0, 2.0 ** -26, -(2.0 ** -27), 1e-300]
    for name in ("sin", "cos", "sinh", "cosh"):
        check(cr, name, np.array(sv + [1e308, -1e308, 1.7976931348623157e308]))
    check(cr, "asin", np.array(sv))
    for name, bad in (("sin", [inf, -inf, nan]), ("cos", [inf, -inf, nan]), ("asin", [inf, -inf, nan, 2.0, -1.5])):
        assert np.all(np.isnan(evaluate(cr, name, np.array(bad)))), name
    assert np.all(np.isnan(evaluate(cr, "sinh", np.array([nan]))))
    assert list(evaluate(cr, "sinh", np.array([inf, -inf, 800.0, -800.0]))) == [inf, -inf, inf, -inf]
    assert list(evaluate(cr, "cosh", np.array([inf, -inf, 800.0, -800.0]))) == [inf, inf, inf, inf]
    pi, pio2, pio4 = math.pi, math.pi / 2, math.pi / 4
    cases = [(0.0, 1.0, 0.0), (-0.0, 1.0, -0.0), (0.0, -1.0, pi), (-0.0, -1.0, -pi), (0.0, 0.0, 0.0),
             (-0.0, 0.0, -0.0), (0.0, -0.0, pi), (-0.0, -0.0, -pi), (1.0, 0.0, pio2), (-1.0, -0.0, -pio2),
             (inf, inf, pio4), (-inf, inf, -pio4), (inf, -inf, 3 * pio4), (-inf, -inf, -3 * pio4),
             (1.0, inf, 0.0), (-1.0, inf, -0.0), (1.0, -inf, pi), (-1.0, -inf, -pi), (inf, 1.0, pio2),
             (-inf, -5.0, -pio2), (1e-310, 1e300, 0.0), (1e300, 1e-310, pio2), (-1e300, -1e-310, -pio2)]
    y = np.array([c[0] for c in cases])
    x = np.array([c[1] for c in cases])
    out = evaluate(cr, "atan2", y, x)
    for (yy, xx, want), g in zip(cases, out):
        assert g == want and math.copysign(1, g) == math.copysign(1, want), (yy, xx, g, want)
    assert np.isnan(evaluate(cr, "atan2", np.array([nan, 1.0]), np.array([1.0, nan]))).all()


def test_sincos_same_bits(cr):
    rng = np.random.default_rng(15)
    a = np.concatenate([rng.uniform(-4, 4, 2000), logu(rng, -30, 30, 2000), [0.0, -0.0, 2.0 ** -27, 1e300]])
    s_ref, c_ref = evaluate(cr, "sin", a), evaluate(cr, "cos", a)
    s, c = ctypes.c_double(), ctypes.c_double()
    for i, v in enumerate(a):
        cr.bmadgpu_cr_sincos(v, ctypes.byref(s), ctypes.byref(c))
        assert s.value == s_ref[i] and c.value == c_ref[i], v


def test_sinhcosh_same_bits(cr):
    rng = np.random.default_rng(16)
    a = np.concatenate([rng.uniform(-3, 3, 2000), rng.uniform(0.2, 0.3, 500), logu(rng, -30, 9.47, 2000),
                        [0.0, -0.0, 0.25, -0.25, 710.0, 711.0, 2.0 ** -26]])
    s_ref, c_ref = evaluate(cr, "sinh", a), evaluate(cr, "cosh", a)
    s, c = ctypes.c_double(), ctypes.c_double()
    for i, v in enumerate(a):
        cr.bmadgpu_cr_sinhcosh(v, ctypes.byref(s), ctypes.byref(c))
        assert s.value == s_ref[i] and c.value == c_ref[i], v


def test_tan(cr):
    rng = np.random.default_rng(17)
    for a in (rng.uniform(-0.8, 0.8, N), rng.uniform(-4, 4, N), rng.uniform(-1e5, 1e5, N),
              logu(rng, -40, 20, N), logu(rng, 20, 1023, N // 3),
              # next to odd multiples of pi/2 (the poles) and to multiples of pi (the zeros)
              np.array([k * math.pi / 2 * (1 + e) for k in range(1, 40) for e in (-3e-16, 0, 3e-16, 1e-12)]),
              np.array([0.0, -0.0, 5e-324, 2.0 ** -27, -(2.0 ** -28), 1e-300])):
        check(cr, "tan", a)
    assert np.all(np.isnan(evaluate(cr, "tan", np.array([math.inf, -math.inf, math.nan]))))


def test_exp(cr):
    rng = np.random.default_rng(18)
    for a in (rng.uniform(-1, 1, N), rng.uniform(-700, 700, N), logu(rng, -60, 0, N),
              rng.uniform(709.0, 709.79, N // 3), rng.uniform(-745.2, -700.0, N),
              np.array([0.0, -0.0, 5e-324, 2.0 ** -54, -(2.0 ** -54), 2.0 ** -53, 1.0, -1.0,
                        709.782712893384, 709.7827128933841, -708.3, -708.39, -745.13, -745.14, -746.0, -800.0])):
        check(cr, "exp", a)
    out = evaluate(cr, "exp", np.array([math.inf, -math.inf, 710.0, math.nan]))
    assert out[0] == math.inf and out[1] == 0.0 and out[2] == math.inf and math.isnan(out[3])

