"""The CPU oracle against the reference's own golden vectors (checker pinning, no GPU)."""
import ctypes
import json
import os

import pytest

from conftest import OracleCoord, load_abi, load_oracle

HERE = os.path.dirname(os.path.abspath(__file__))


def _printed_tol(x, digits):
    # Golden values are printed with `digits` significant digits: allow half a unit in the last one.
    if x == 0:
        return 0.0
    import math
    e = math.floor(math.log10(abs(x)))
    return 0.5 * 10.0 ** (e - digits + 1)


def _tm_cases():
    return json.load(open(os.path.join(HERE, "golden", "tracking_method_bmad_standard.json")))


@pytest.mark.parametrize("case", _tm_cases()["cases"], ids=lambda c: c["name"])
def test_tracking_method_bmad_standard(case):
    abi, lib = load_abi(), load_oracle()
    data = _tm_cases()
    p = abi.electron_param(data["e_tot"], charge=data["charge"])
    ele = abi.default_element(getattr(abi, case["key"]), **case["attrs"])
    c = OracleCoord()
    start = (ctypes.c_double * 6)(*data["start"])
    lib.oracle_init_coord(ctypes.byref(c), start, ctypes.byref(p))
    err = lib.oracle_track1(ctypes.byref(c), ctypes.byref(ele), 1, ctypes.byref(p))
    assert err == 0
    assert c.state == abi.ALIVE
    for i in range(6):
        want = case["expected_vec"][i]
        tol = case["tol"] + _printed_tol(want, 11)
        assert abs(c.vec[i] - want) <= tol, (case["name"], i, c.vec[i], want)


def test_fringe_test_hwang():
    abi, lib = load_abi(), load_oracle()
    data = json.load(open(os.path.join(HERE, "golden", "fringe_test_hwang.json")))
    p = abi.electron_param(data["e_tot"], charge=data["charge"])
    ele = abi.default_element(abi.SBEND, l=0.0, **data["element"])
    for case in data["cases"]:
        c = OracleCoord()
        start = (ctypes.c_double * 6)(*data["start"])
        lib.oracle_init_coord(ctypes.byref(c), start, ctypes.byref(p))
        mat = (ctypes.c_double * 36)(*[1.0 if i % 7 == 0 else 0.0 for i in range(36)])
        at = 11 if case["edge"] == "first_track_edge" else 12
        assert lib.oracle_hwang_bend_edge_kick(ctypes.byref(ele), ctypes.byref(p), at, ctypes.byref(c), mat) == 0
        for i in range(6):
            want = case["expected_dorb"][i]
            got = c.vec[i] - data["start"][i]
            assert abs(got - want) <= case["tol"] + _printed_tol(want, 7), (case["edge"], i, got, want)
        for i in range(6):
            for j in range(6):
                want = case["expected_dmat"][i][j]
                got = mat[i * 6 + j] - (1.0 if i == j else 0.0)
                assert abs(got - want) <= case["tol"] + _printed_tol(want, 7), (case["edge"], i, j, got, want)
