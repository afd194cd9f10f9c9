"""Closed orbit, one-turn matrix, periodic Twiss and the matched beam on the GPU:

  - the one-turn matrix from device tracking equals the one the same stencil gives on the
    oracle's tracking;
  - the closed orbit (dims 4, 5, 6, ideal and misaligned rings) is a fixed point of the ORACLE's
    one-turn map to the reference's stopping rule, and equals the oracle-restated Newton result;
  - the Twiss of the device matrix equals the restatement's on the oracle matrix;
  - the beam generator's deviates are the numpy Philox4x32-10 / Box-Muller stream; the beam built
    from given deviates equals the numpy restatement of init_bunch_distribution; at full size the
    renormalised beam has exactly the target centroid and covariance (size-independent property)."""
import importlib
import math

import numpy as np
import pytest

import optics_reference as R
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


RINGS = {"ideal": lambda: rings.ring(50), "misaligned": lambda: rings.perturbed_ring(50, seed=3),
         "misaligned7": lambda: rings.perturbed_ring(100, seed=7, offset_sigma=100e-6)}


@pytest.mark.parametrize("rf_on", [False, True])
def test_one_turn_matrix_matches_oracle(ctx, rf_on):
    eles, p = rings.perturbed_ring(50, seed=3)
    lat = lib.Lattice(ctx, eles, p)
    orbit = np.array([1e-4, -2e-5, 5e-5, 1e-5, 1e-4, 2e-4])
    M, end = lib.one_turn_matrix(ctx, lat, orbit, rf_on=rf_on)
    arr, pp = R.orbit_lattice(eles, p, rf_off=not rf_on)
    f, Mo = R.one_turn(arr, pp, orbit)
    assert np.allclose(end, f, rtol=1e-12, atol=1e-16)
    assert np.max(np.abs(M - Mo)) < 1e-9 * max(1.0, np.max(np.abs(Mo)))
    S = np.zeros((4, 4))
    S[0, 1] = S[2, 3] = 1.0
    S[1, 0] = S[3, 2] = -1.0
    if not rf_on:  # the transverse block of the RF-off map is symplectic (to the stencil's accuracy)
        assert np.max(np.abs(M[:4, :4].T @ S @ M[:4, :4] - S)) < 1e-8


@pytest.mark.parametrize("ring", list(RINGS))
@pytest.mark.parametrize("dim", [4, 5, 6])
def test_closed_orbit_is_oracle_fixed_point(ctx, ring, dim):
    eles, p = RINGS[ring]()
    lat = lib.Lattice(ctx, eles, p)
    guess = np.zeros(6)
    if dim == 4:
        guess[5] = 1e-3  # transverse orbit at a fixed energy offset
    x, M, it = lib.closed_orbit(ctx, lat, dim=dim, guess=guess)
    assert it < 20
    # fixed point of the oracle's map, to the reference's rule (rel 1e-9, abs 1e-12) with margin
    arr, pp = R.orbit_lattice(eles, p, rf_off=(dim != 6))
    f = oracle_track(arr, pp, x[:, None], 1)["vec"][:, 0]
    n_fit = dim
    assert np.all(np.abs(f[:n_fit] - x[:n_fit]) < 2 * (np.abs(x[:n_fit]) * 1e-9 + 1e-12)), (f - x)
    if dim != 6:
        assert x[4] == 0.0
    if dim == 4:
        assert x[5] == 1e-3
    # the oracle-restated Newton converges to the same fixed point
    xo, Mo = R.closed_orbit(eles, p, dim, guess=guess)
    assert np.all(np.abs(x - xo) <= 1e-8 * np.abs(xo) + 1e-10), (x, xo)
    assert np.max(np.abs(M - Mo)) < 1e-8 * max(1.0, np.max(np.abs(Mo)))


@pytest.mark.parametrize("ring", list(RINGS))
def test_twiss_matches_oracle_matrix(ctx, ring):
    eles, p = RINGS[ring]()
    lat = lib.Lattice(ctx, eles, p)
    x, _, _ = lib.closed_orbit(ctx, lat, dim=6)
    M, _ = lib.one_turn_matrix(ctx, lat, x, rf_on=False)  # twiss_at_start's RF-off matrix
    got = lib.twiss_from_mat6(M, x)
    arr, pp = R.orbit_lattice(eles, p, rf_off=True)
    _, Mo = R.one_turn(arr, pp, x)
    want = R.twiss_from_mat6(Mo, x)
    assert got["status"] == want["status"] == lib.TWISS_OK
    for k in ("beta_a", "alpha_a", "phi_a", "beta_b", "alpha_b", "phi_b", "eta_x", "etap_x", "eta_a", "eta_b",
              "gamma_c"):
        assert abs(got[k] - want[k]) <= 1e-8 * max(1.0, abs(want[k])), (k, got[k], want[k])
    if ring == "ideal":
        lin = rings.periodic_optics(eles)
        assert got["beta_a"] == pytest.approx(lin["beta_a"], rel=1e-8)
        assert got["phi_b"] / (2 * math.pi) == pytest.approx(lin["tune_b"], abs=1e-9)


def test_closed_orbit_argument_errors(ctx):
    eles, p = rings.ring(10, rf=False)
    lat = lib.Lattice(ctx, eles, p)
    with pytest.raises(lib.BmadGpuError):
        lib.closed_orbit(ctx, lat, dim=6)       # no RF voltage
    with pytest.raises(lib.BmadGpuError):
        lib.closed_orbit(ctx, lat, dim=3)
    x, _, _ = lib.closed_orbit(ctx, lat)      # default dim: 4 without RF
    assert np.all(x == 0)


def test_deviates_match_restatement(ctx):
    for cut in (0.0, 2.0):
        got = lib.gaussian_deviates(ctx, seed=0x1234_5678_9ABC, n=5000, sigma_cutoff=cut)
        want = R.deviates(0x1234_5678_9ABC, 5000, sigma_cutoff=cut)
        assert np.max(np.abs(got - want)) < 1e-13
        if cut:
            assert np.max(np.abs(got)) <= cut


BEAM = dict(a_emit=2e-9, b_emit=20e-12, sig_z=4e-3, sig_pz=8e-4, dpz_dz=0.05)


@pytest.mark.parametrize("ring", ["ideal", "misaligned"])
@pytest.mark.parametrize("renorm", [True, False])
def test_beam_matches_restatement(ctx, ring, renorm):
    eles, p = RINGS[ring]()
    lat = lib.Lattice(ctx, eles, p)
    x, _, _ = lib.closed_orbit(ctx, lat, dim=6)
    M, _ = lib.one_turn_matrix(ctx, lat, x, rf_on=False)
    tw = lib.twiss_from_mat6(M, x)
    n = 20000
    normals = R.deviates(99, n)
    center = [1e-5, 0, -2e-5, 0, 0, 1e-5]
    hb = lib.beam_init_gaussian(ctx, p, tw, n, normals=normals, center=center, orbit=x, renorm_center=renorm,
                                renorm_sigma=renorm, sig_z_jitter=0.01, center_jitter=[1e-6] * 6, **BEAM)
    want = R.init_random_distribution(normals, n, tw, center=center, orbit=x, renorm_center=renorm,
                                      renorm_sigma=renorm, sig_z_jitter=0.01, center_jitter=[1e-6] * 6, **BEAM)
    sig = np.std(want, axis=1)
    assert np.max(np.abs(hb.vec - want) / sig[:, None]) < 1e-12
    assert np.all(hb.state == abi.ALIVE)
    pc = p.p0c * (1 + hb.vec[5])
    assert np.allclose(hb.beta, pc / np.sqrt(pc * pc + p.mass ** 2), rtol=1e-15)
    assert np.allclose(hb.t, -hb.vec[4] / (hb.beta * abi.C_LIGHT), rtol=1e-15)


def test_beam_full_size_exact_moments(ctx):
    """1M particles drawn on the device: with renormalisation the centroid is the closed orbit
    and the normal-mode covariance is exactly the target (sigma_ij from the Twiss), whatever the
    sample."""
    eles, p = rings.perturbed_ring(50, seed=3)
    lat = lib.Lattice(ctx, eles, p)
    x, _, _ = lib.closed_orbit(ctx, lat, dim=6)
    M, _ = lib.one_turn_matrix(ctx, lat, x, rf_on=False)
    tw = lib.twiss_from_mat6(M, x)
    n = 1 << 20
    hb = lib.beam_init_gaussian(ctx, p, tw, n, seed=2024, orbit=x, **BEAM)
    v = hb.vec - x[:, None]
    assert np.max(np.abs(v.mean(axis=1)) / np.std(v, axis=1)) < 1e-12
    # undo coupling and dispersion: normal-mode coordinates
    C = np.asarray(tw["c_mat"]).reshape(2, 2)
    g = tw["gamma_c"]
    Vinv = np.zeros((4, 4))
    Vinv[:2, :2] = Vinv[2:, 2:] = g * np.eye(2)
    Vinv[:2, 2:] = -C
    Vinv[2:, :2] = R.symp_conj(C)
    a = Vinv @ v[:4]
    a = a - np.outer([tw["eta_a"], tw["etap_a"], tw["eta_b"], tw["etap_b"]], v[5])
    emit_a = math.sqrt(np.mean(a[0] ** 2) * np.mean(a[1] ** 2) - np.mean(a[0] * a[1]) ** 2)
    emit_b = math.sqrt(np.mean(a[2] ** 2) * np.mean(a[3] ** 2) - np.mean(a[2] * a[3]) ** 2)
    assert emit_a == pytest.approx(BEAM["a_emit"], rel=1e-10)
    assert emit_b == pytest.approx(BEAM["b_emit"], rel=1e-10)
    assert np.mean(a[0] ** 2) / emit_a == pytest.approx(tw["beta_a"], rel=1e-10)
    assert np.std(v[4]) == pytest.approx(BEAM["sig_z"], rel=1e-10)
    assert np.std(v[5]) == pytest.approx(BEAM["sig_pz"], rel=1e-10)
    assert np.mean(v[4] * v[5]) / np.var(v[4]) == pytest.approx(BEAM["dpz_dz"], rel=1e-9)
    # seeded: the same seed gives the same beam bit for bit
    hb2 = lib.beam_init_gaussian(ctx, p, tw, n, seed=2024, orbit=x, **BEAM)
    assert np.array_equal(hb.vec, hb2.vec)


@pytest.mark.parametrize("n", [1, 2, 5, 7])
def test_beam_small_counts_match_restatement(ctx, n):
    """The reference's special cases: one particle (no renormalisation at all), up to six (only
    the diagonal normalised, no shears), seven (the first count with the shears)."""
    eles, p = rings.ring(20)
    lat = lib.Lattice(ctx, eles, p)
    x, _, _ = lib.closed_orbit(ctx, lat, dim=6)
    tw = lib.twiss_from_mat6(lib.one_turn_matrix(ctx, lat, x, rf_on=False)[0], x)
    normals = R.deviates(31 + n, n)
    hb = lib.beam_init_gaussian(ctx, p, tw, n, normals=normals, orbit=x, **BEAM)
    want = R.init_random_distribution(normals, n, tw, orbit=x, **BEAM)
    scale = np.array([1e-4, 1e-5, 1e-5, 1e-6, 1e-3, 1e-3])[:, None]
    assert np.max(np.abs(hb.vec - want) / scale) < 1e-10, (hb.vec, want)
    if n == 1:  # a single particle, re-centred: the closed orbit itself
        assert np.allclose(hb.vec[:, 0], x, rtol=0, atol=1e-18)
