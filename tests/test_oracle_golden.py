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


# ---- transfer matrices by tracking (mat6_calc_method_test) ---------------------------------------

def _m6_cases():
    return json.load(open(os.path.join(HERE, "golden", "mat6_calc_method_tracking.json")))


# Elements whose edge kicks the oracle does not restate (fringe_type full: exact_bend_edge_kick,
# hard_multipole_edge_kick, soft_quadrupole_edge_kick); the oracle refuses them.
M6_NOT_RESTATED = set()


def matrix_by_tracking(track, start, d):
    """make_mat6_tracking (bmad/low_level/make_mat6_tracking.f90:26-110): the central particle and
    the twelve particles displaced by +-d in one coordinate, tracked through the element; column i
    of the matrix is the difference of the two end orbits over 2 d, and vec0 = end - matrix start.
    track(list of 6-vectors) -> (list of end 6-vectors, list of states)."""
    import numpy as np
    starts = [list(start)]
    for i in range(6):
        for sgn in (1, -1):
            v = list(start)
            v[i] = v[i] + sgn * d
            starts.append(v)
    ends, states = track(starts)
    ends = np.asarray(ends, dtype=np.float64)
    assert all(s == 1 for s in states), states
    mat = np.empty((6, 6))
    for i in range(6):
        mat[:, i] = (ends[1 + 2 * i] - ends[2 + 2 * i]) / (2 * d)
    vec0 = ends[0] - mat @ np.asarray(start)
    return mat, vec0


def _oracle_tracker(abi, lib, ele, p):
    def track(starts):
        ends, states = [], []
        for v in starts:
            c = OracleCoord()
            lib.oracle_init_coord(ctypes.byref(c), (ctypes.c_double * 6)(*v), ctypes.byref(p))
            assert lib.oracle_track1(ctypes.byref(c), ctypes.byref(ele), 1, ctypes.byref(p)) == 0
            ends.append([c.vec[i] for i in range(6)])
            states.append(c.state)
        return ends, states
    return track


@pytest.mark.parametrize("case", _m6_cases()["cases"], ids=lambda c: c["name"])
def test_mat6_by_tracking(case):
    """The oracle's transfer matrix and vec0 by central differences against the reference's
    "Tracking" lines of mat6_calc_method_test (ABS 1e-9 on every entry)."""
    import numpy as np
    if case["name"] in M6_NOT_RESTATED:
        pytest.skip("edge kick of fringe_type full not restated")
    abi, lib = load_abi(), load_oracle()
    data = _m6_cases()
    p = abi.electron_param(data["e_tot"], charge=data["charge"])
    ele = abi.default_element(getattr(abi, case["key"]), **case["attrs"])
    mat, vec0 = matrix_by_tracking(_oracle_tracker(abi, lib, ele, p), data["start"], data["d_orb"])
    want = np.asarray(case["expected_mat6"])
    tol = np.asarray(case["tol_rows"])[:, None] + 5e-14 * np.abs(want)
    bad = np.argwhere(np.abs(mat - want) > tol)
    assert bad.size == 0, (case["name"], [(tuple(ij), mat[tuple(ij)], want[tuple(ij)]) for ij in bad[:4]])
    want0 = np.asarray(case["expected_vec0"])
    assert np.all(np.abs(vec0 - want0) <= case["tol_vec0"] + 5e-14 * np.abs(want0)), (case["name"], vec0, want0)


# ---- collimator apertures (aperture_test) --------------------------------------------------------

def _ap_cases():
    return json.load(open(os.path.join(HERE, "golden", "aperture_test_collimators.json")))["cases"]


def _printed3(x):
    import math
    return 0.0 if x == 0 else 0.5 * 10.0 ** (math.floor(math.log10(abs(x))) - 2)


@pytest.mark.parametrize("case", _ap_cases(), ids=lambda c: c["name"])
def test_aperture_test_collimators(case):
    """check_aperture_limit at the exit of the reference's ecollimator / rcollimator on each 9-point
    grid: the states (S lines) exactly, param%unstable_factor (U lines, printed with 3 digits)."""
    abi, lib = load_abi(), load_oracle()
    p = abi.electron_param(3.1e9, charge=1.0)
    ele = abi.default_element(getattr(abi, case["key"]), **case["attrs"])
    for v, want_state, want_u in zip(case["vecs"], case["expected_state"], case["expected_unstable"]):
        c = OracleCoord()
        lib.oracle_init_coord(ctypes.byref(c), (ctypes.c_double * 6)(*v), ctypes.byref(p))
        u = ctypes.c_double()
        assert lib.oracle_check_aperture(ctypes.byref(ele), ctypes.byref(p), 12, ctypes.byref(c), ctypes.byref(u)) == 0
        assert c.state == want_state, (case["name"], v, c.state, want_state)
        assert abs(u.value - want_u) <= case["tol"] + _printed3(want_u), (case["name"], v, u.value, want_u)


# ---- offset_particle of bends (coord_test) ------------------------------------------------------

def _ct():
    return json.load(open(os.path.join(HERE, "golden", "coord_test_bend_offsets.json")))


@pytest.mark.parametrize("case", _ct()["cases"], ids=lambda c: c["name"])
def test_coord_test_bend_offsets(case):
    """offset_particle set, track1 through the unmisaligned bend, offset_particle unset, for the
    reference's b0 / b1 (offsets, pitches, roll) / b2 (also ref_tilt) against its coord_test
    lines (8 printed decimals, ABS 1e-8)."""
    abi, lib = load_abi(), load_oracle()
    data = _ct()
    p = abi.electron_param(data["e_tot"], charge=data["charge"])
    ele = abi.default_element(abi.SBEND, **case["attrs"])
    bare = dict(case["attrs"])
    for k in ("x_offset", "y_offset", "x_pitch", "y_pitch", "roll", "ref_tilt", "z_offset"):
        bare.pop(k, None)
    ele2 = abi.default_element(abi.SBEND, **bare)   # zero_ele_offsets
    c = OracleCoord()
    lib.oracle_init_coord(ctypes.byref(c), (ctypes.c_double * 6)(*case["start"]), ctypes.byref(p))
    tol = case["tol"] + 5e-9

    def check(stage):
        want = case["expected"][stage]
        got = [c.vec[i] for i in range(6)]
        assert all(abs(g - w) <= tol for g, w in zip(got, want)), (case["name"], stage, got, want)

    assert lib.oracle_offset_particle(ctypes.byref(ele), ctypes.byref(p), 1, ctypes.byref(c)) == 0
    check("In:")
    assert lib.oracle_track1(ctypes.byref(c), ctypes.byref(ele2), 1, ctypes.byref(p)) == 0
    check("Xfer")
    assert lib.oracle_offset_particle(ctypes.byref(ele), ctypes.byref(p), 0, ctypes.byref(c)) == 0
    check("Out")
