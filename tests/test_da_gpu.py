"""Dynamic-aperture search on the GPU (bmadgpu_da_scan): every ray's bisection, run for all
rays at once with the search state on the device, against the same search (restated from
dynamic_aperture_point, bmad/modules/dynamic_aperture_mod.f90:284-398) driven by the oracle's
tracking one trial particle at a time. The survive/lost outcome of each trial decides the whole
sequence of trial points, so the two searches agree exactly unless a trial lands where the GPU's
and glibc's last-bit differences flip the outcome; then they may differ by the final accuracy."""
import importlib
import math

import numpy as np
import pytest

from conftest import load_abi
from helpers import oracle_track

pytestmark = pytest.mark.gpu
lib = importlib.import_module("bmad-ecosystem_b200.lib")
rings = importlib.import_module("bmad-ecosystem_b200.rings")
abi = load_abi()


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    yield c
    c.close()


def oracle_da_point(eles, p, theta, n_turn, x_init, y_init, abs_acc, rel_acc, orb0):
    x0 = y0 = 0.0
    x1, y1 = math.cos(theta) * x_init, math.sin(theta) * y_init
    x2 = y2 = 0.0
    bracketed, turn_lost, ix_ele, plane = False, 0, -1, 0
    for _ in range(200):
        v = np.array(orb0, float).reshape(6, 1).copy()
        v[0, 0] += x1
        v[2, 0] += y1
        o = oracle_track(eles, p, v, n_turn)
        if o["state"][0] != abi.ALIVE:
            x2, y2 = x1, y1
            turn_lost, ix_ele, plane, bracketed = int(o["ix_turn"][0]) + 1, int(o["ix_ele"][0]), int(o["state"][0]), True
        else:
            x0, y0 = x1, y1
        if bracketed:
            x1, y1 = (x0 + x2) / 2, (y0 + y2) / 2
        else:
            x1, y1 = 2 * x1, 2 * y1
        if bracketed:
            r = 0.5 * math.sqrt((x0 + x2) ** 2 + (y0 + y2) ** 2)
            if math.sqrt((x2 - x0) ** 2 + (y2 - y0) ** 2) <= 2 * (abs_acc + r * rel_acc):
                break
    return dict(x=x1, y=y1, i_turn=turn_lost, ix_ele=ix_ele, plane=plane)


def test_da_scan_matches_oracle_search(ctx):
    eles, p = rings.ring(50)
    lat = lib.Lattice(ctx, eles, p)
    theta = np.linspace(0.05, math.pi - 0.05, 9)
    orb0 = np.zeros((len(theta), 6))
    orb0[1::3, 5] = 0.005            # some rays off momentum
    kw = dict(n_turn=64, x_init=1e-3, y_init=1e-3, abs_accuracy=2e-5, rel_accuracy=1e-3)
    got = lib.da_scan(ctx, lat, theta, orb0=orb0, **kw)
    exact = 0
    for i, th in enumerate(theta):
        want = oracle_da_point(eles, p, th, kw["n_turn"], kw["x_init"], kw["y_init"], kw["abs_accuracy"],
                               kw["rel_accuracy"], orb0[i])
        g = got[i]
        tol = 2 * (kw["abs_accuracy"] + math.hypot(want["x"], want["y"]) * kw["rel_accuracy"])
        assert math.hypot(g["x"] - want["x"], g["y"] - want["y"]) <= tol, (i, g, want)
        if g["x"] == want["x"] and g["y"] == want["y"]:
            exact += 1
            assert (g["i_turn"], g["ix_ele"], g["plane"]) == (want["i_turn"], want["ix_ele"], want["plane"])
        assert g["plane"] in (abi.LOST_NEG_X, abi.LOST_POS_X, abi.LOST_NEG_Y, abi.LOST_POS_Y, abi.LOST_PZ, abi.LOST)
    assert exact >= len(theta) - 1


def test_da_scan_arguments(ctx):
    eles, p = rings.ring(10)
    lat = lib.Lattice(ctx, eles, p)
    with pytest.raises(lib.BmadGpuError) as ex:
        lib.da_scan(ctx, lat, [0.3], n_turn=8, x_init=0.0)
    assert ex.value.code == abi.EINVAL
    assert lib.da_scan(ctx, lat, [], n_turn=8) == []
