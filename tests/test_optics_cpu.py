"""Optics set-up on the host (no GPU): the Twiss of a one-turn matrix (bmadgpu_twiss_from_mat6)
against the numpy restatement of twiss_from_mat6 / mat_symp_decouple / twiss_from_mat2, the
closed orbit and one-turn matrix restated on the oracle's tracking against the analytic linear
optics, and the Philox4x32-10 block function of the beam generator against the published
known-answer vectors."""
import importlib
import math

import numpy as np
import pytest

import optics_reference as R

lib = importlib.import_module("bmad-ecosystem_b200.lib")
rings = importlib.import_module("bmad-ecosystem_b200.rings")

FIELDS = ("beta_a", "alpha_a", "gamma_a", "phi_a", "beta_b", "alpha_b", "gamma_b", "phi_b", "eta_x", "etap_x",
          "eta_y", "etap_y", "eta_a", "etap_a", "eta_b", "etap_b", "gamma_c")


def rot2(mu, beta, alpha):
    g = (1 + alpha ** 2) / beta
    c, s = math.cos(mu), math.sin(mu)
    return np.array([[c + alpha * s, beta * s], [-g * s, c - alpha * s]])


def coupled_matrix(theta=0.07):
    """A stable, coupled, symplectic one-turn matrix: an uncoupled one conjugated by a rotation
    of the x-y plane, with a dispersion column."""
    U = np.zeros((4, 4))
    U[:2, :2] = rot2(2 * math.pi * 0.31, 8.0, -0.4)
    U[2:, 2:] = rot2(2 * math.pi * 0.17, 3.0, 0.6)
    c, s = math.cos(theta), math.sin(theta)
    Rm = np.array([[c, 0, s, 0], [0, c, 0, s], [-s, 0, c, 0], [0, -s, 0, c]])
    m6 = np.eye(6)
    m6[:4, :4] = Rm @ U @ Rm.T
    m6[:4, 5] = [0.3, 0.02, 0.01, -0.004]
    return m6


@pytest.mark.parametrize("case", ["uncoupled", "coupled", "coupled_strong"])
def test_twiss_matches_restatement(case):
    if case == "uncoupled":
        m6 = np.eye(6)
        m6[:2, :2] = rot2(2.2, 12.0, 1.3)
        m6[2:4, 2:4] = rot2(1.1, 4.0, -0.2)
        m6[:2, 5] = [0.7, 0.05]
    else:
        m6 = coupled_matrix(0.07 if case == "coupled" else 0.4)
    got = lib.twiss_from_mat6(m6, [1e-4, -2e-5, 3e-5, 1e-6, 0, 1e-3])
    want = R.twiss_from_mat6(m6)
    assert got["status"] == want["status"] == lib.TWISS_OK
    for k in FIELDS:
        assert abs(got[k] - want[k]) <= 1e-13 * max(1.0, abs(want[k])), (k, got[k], want[k])
    assert np.allclose(got["c_mat"], want["c_mat"], rtol=0, atol=1e-14)
    if case == "uncoupled":
        assert got["beta_a"] == pytest.approx(12.0, rel=1e-13)
        assert got["phi_b"] == pytest.approx(1.1, rel=1e-13)
        assert got["gamma_c"] == 1.0


def test_twiss_status_codes():
    m6 = np.eye(6)
    m6[:2, :2] = [[2.0, 1.0], [1.0, 1.0]]      # |trace| > 2: a mode unstable
    m6[2:4, 2:4] = rot2(1.0, 3.0, 0.0)
    assert lib.twiss_from_mat6(m6)["status"] == R.twiss_from_mat6(m6)["status"] == lib.TWISS_UNSTABLE_A
    m6[:2, :2] = [[3.0, 1.0], [0.0, 1.0]]      # det 3: far from symplectic
    assert lib.twiss_from_mat6(m6)["status"] == R.twiss_from_mat6(m6)["status"] == lib.TWISS_NON_SYMPLECTIC
    m6 = np.eye(6) * 1e11
    assert lib.twiss_from_mat6(m6)["status"] == lib.TWISS_UNSTABLE


def test_oracle_orbit_optics_match_linear_optics():
    """The closed orbit and one-turn matrix restated on the oracle's tracking give, for the ideal
    ring, the zero orbit and the Twiss of the product of the linear element matrices."""
    eles, p = rings.ring(20)
    x, M = R.closed_orbit(eles, p, 4)
    assert np.all(np.abs(x) < 1e-15)
    tw = lib.twiss_from_mat6(M, x)
    lin = rings.periodic_optics(eles)
    for a, b in (("beta_a", "beta_a"), ("alpha_a", "alpha_a"), ("beta_b", "beta_b"), ("alpha_b", "alpha_b"),
                 ("eta_x", "eta_x"), ("etap_x", "etap_x")):
        assert tw[a] == pytest.approx(lin[b], rel=1e-8, abs=1e-9), a
    assert tw["phi_a"] / (2 * math.pi) == pytest.approx(lin["tune_a"], abs=1e-9)


# Random123's known-answer vectors for philox4x32_10 (counter, key, result).
KAT = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
       ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
       ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
        (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]


@pytest.mark.parametrize("ctr,key,want", KAT)
def test_philox_known_answers(ctr, key, want):
    assert tuple(lib.philox4x32_10(ctr, key)) == want
    got = R.philox4x32_10(*[np.array([v], np.uint64) for v in ctr], *key)
    assert tuple(int(v[0]) for v in got) == want
