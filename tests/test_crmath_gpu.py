"""The correctly rounded transcendentals on the device (bmadgpu_cr_eval) against their host
build, bit for bit, on a million arguments per function over the ranges the maps use and far
beyond; the host build is checked against mpmath on the CPU (tests/test_crmath_cpu.py), and a
sample of the device results against mpmath here."""
import ctypes
import importlib

import numpy as np
import pytest

import test_crmath_cpu as H

pytestmark = pytest.mark.gpu
lib = importlib.import_module("bmad-ecosystem_b200.lib")
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    yield c
    c.close()


def device_eval(ctx, fn, a, b=None):
    so = lib.load()
    so.bmadgpu_cr_eval.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_int64]
    da = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
    db = torch.from_numpy(np.ascontiguousarray(b if b is not None else a, dtype=np.float64)).cuda()
    out = torch.empty(2 * len(a), dtype=torch.float64, device="cuda")
    lib.check(so.bmadgpu_cr_eval(ctx.handle, fn, da.data_ptr(), db.data_ptr(), out.data_ptr(), len(a)))
    return out.cpu().numpy()


def arguments(name, rng, n):
    lu = lambda lo, hi, m: np.exp2(rng.uniform(lo, hi, m)) * rng.choice([-1.0, 1.0], m)
    if name in ("sin", "cos"):
        return np.concatenate([rng.uniform(-0.8, 0.8, n), rng.uniform(-4, 4, n), lu(-60, 30, n), lu(20, 1023, n // 8),
                               [0.0, -0.0, 5e-324, np.inf, -np.inf, np.nan]])
    if name == "asin":
        return np.concatenate([rng.uniform(-1, 1, n), lu(-60, 0, n), rng.uniform(-1e-3, 1e-3, n),
                               [1.0, -1.0, 0.0, -0.0, 2.0, np.nan]])
    if name == "atan2":
        return np.concatenate([lu(-60, 60, n), rng.uniform(-1, 1, n), lu(-1000, 1000, n // 8), [0.0, -0.0, np.inf]])
    if name == "tan":
        return np.concatenate([rng.uniform(-0.8, 0.8, n), rng.uniform(-4, 4, n), lu(-60, 30, n), lu(20, 1023, n // 8),
                               [0.0, -0.0, 5e-324, np.inf, -np.inf, np.nan, np.pi / 2]])
    if name == "exp":
        return np.concatenate([rng.uniform(-1, 1, n), rng.uniform(-745, 709.7, n), lu(-60, -20, n),
                               [0.0, -0.0, np.inf, -np.inf, np.nan, 2.0 ** -53, -708.39, 709.78]])
    return np.concatenate([rng.uniform(-0.3, 0.3, n), rng.uniform(-3, 3, n), rng.uniform(-711, 711, n),
                           lu(-60, 0, n), [0.0, -0.0, np.inf, -np.inf, np.nan, 2.0 ** -26]])


def same_bits(x, y):
    """Equal bit patterns, NaNs of any payload counting as equal."""
    nx, ny = np.isnan(x), np.isnan(y)
    return np.array_equal(nx, ny) and np.array_equal(x[~nx].view(np.uint64), y[~ny].view(np.uint64))


@pytest.mark.parametrize("name", ["sin", "cos", "asin", "atan2", "sinh", "cosh", "exp", "tan"])
def test_device_equals_host_build(ctx, cr_host, name):
    rng = np.random.default_rng(100 + H.FN[name])
    a = arguments(name, rng, 250000)
    b = arguments("atan2", np.random.default_rng(7), 250000)[:len(a)] if name == "atan2" else None
    if b is not None and len(b) < len(a):
        b = np.resize(b, len(a))
    got = device_eval(ctx, H.FN[name], a, b)[:len(a)]
    want = H.evaluate(cr_host, name, a, b)
    assert same_bits(got, want), np.flatnonzero((got.view(np.uint64) != want.view(np.uint64)) & ~np.isnan(want))[:5]
    # a sample straight against mpmath
    for i in np.random.default_rng(3).choice(len(a), 300, replace=False):
        if np.isnan(a[i]) or (b is not None and np.isnan(b[i])):
            continue
        w = H.exact(name, a[i], 0.0 if b is None else b[i])
        assert got[i] == w or (np.isnan(got[i]) and np.isnan(w)), (a[i], got[i], w)


@pytest.mark.parametrize("fn,pair", [(6, ("sin", "cos")), (7, ("sinh", "cosh"))])
def test_fused_pairs_equal_single_functions(ctx, fn, pair):
    rng = np.random.default_rng(fn)
    a = np.concatenate([rng.uniform(-4, 4, 200000), np.exp2(rng.uniform(-40, 9.4, 200000))])
    out = device_eval(ctx, fn, a)
    n = len(a)
    assert same_bits(out[:n], device_eval(ctx, H.FN[pair[0]], a)[:n])
    assert same_bits(out[n:], device_eval(ctx, H.FN[pair[1]], a)[:n])


@pytest.fixture(scope="module")
def cr_host():
    import ctypes as C
    import os
    import subprocess
    if not os.path.exists(H.LIB):
        subprocess.check_call(["make", "-s", "-C", os.path.join(H.ROOT, "bmad-ecosystem_b200", "csrc"), "hostcheck-lib"])
    so = C.CDLL(H.LIB)
    D = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    so.bmadgpu_cr_eval_host.argtypes = [C.c_int, D, D, D, C.c_long]
    return so
