"""Frequency-map analysis on the GPU (bmadgpu_fma): per-particle tunes of the first and last
fft_turns turns equal the numpy restatement of frequency_map's calculation on the oracle's
turn-by-turn tracking; small amplitudes give the ring's linear tunes (the reference's 1 - Q
convention); particles lost or pushed out of the RF bucket are reported as the reference does."""
import importlib
import math

import numpy as np
import pytest

import fma_reference as F

pytestmark = pytest.mark.gpu
lib = importlib.import_module("bmad-ecosystem_b200.lib")
rings = importlib.import_module("bmad-ecosystem_b200.rings")


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    yield c
    c.close()


def grid(n_x=5, n_y=4, x_max=0.011, y_max=0.005, pz=(0.0, 0.002)):
    off = []
    for d in pz:
        for iy in range(n_y):
            for ix in range(n_x):
                off.append([x_max * (ix + 1) / n_x, 0, y_max * (iy + 1) / n_y, 0, 0, d])
    return np.array(off)


@pytest.mark.parametrize("ring,n_turn,fft_turns", [("ideal", 256, 0), ("misaligned", 300, 128), ("ideal", 250, 0),
                                                   ("misaligned", 300, 96)])
def test_fma_matches_restatement(ctx, ring, n_turn, fft_turns):
    eles, p = rings.ring(20) if ring == "ideal" else rings.perturbed_ring(20, seed=5)
    lat = lib.Lattice(ctx, eles, p)
    orbit = lib.closed_orbit(ctx, lat)[0]
    M, _ = lib.one_turn_matrix(ctx, lat, orbit, rf_on=True)
    norm = lib.fma_normalization(M)
    tw = lib.twiss_from_mat6(lib.one_turn_matrix(ctx, lat, orbit, rf_on=False)[0], orbit)
    qa, qb = tw["phi_a"] / (2 * math.pi), tw["phi_b"] / (2 * math.pi)
    off = grid()
    q, st, tl, _ = lib.fma(ctx, lat, off, n_turn, fft_turns=fft_turns, orbit=orbit, norm=norm, tunes=(qa, qb))
    z_limit = 0.25 * 299792458.0 / rings.RF_FREQUENCY
    hist, st_o = F.record(eles, p, (orbit[None, :] + off).T, n_turn, norm, orbit, z_limit)
    assert np.array_equal(st, st_o)
    assert np.sum(st == 0) >= len(off) // 2
    N = fft_turns or n_turn // 2
    want = F.tunes(hist, N, qa < 0.5, qb < 0.5)
    ok = st == 0
    assert np.max(np.abs(q[ok] - want[ok])) < 1e-9


def test_fma_small_amplitude_gives_eigen_tunes(ctx):
    """At small amplitude the tunes are the one-turn matrix's eigen-tunes, in the reference's
    convention: the x and y spectra peak at 1 - Q (z at Q), calc_tune reads bin k as (k + 1) / N (a bias of one bin,
    1/N, that the reference carries), and x/y are flipped back when the ring tune is below 0.5."""
    eles, p = rings.ring(20)
    lat = lib.Lattice(ctx, eles, p)
    orbit = lib.closed_orbit(ctx, lat)[0]
    M, _ = lib.one_turn_matrix(ctx, lat, orbit, rf_on=True)
    vals, _ = lib.mat_eigen(M)
    # peak positions: 1 - Q for x + i px and y + i py, Q for z - i pz
    raw = [1.0 - (np.angle(vals[k]) / (2 * math.pi)) % 1.0 for k in (0, 2)] + [(np.angle(vals[4]) / (2 * math.pi)) % 1.0]
    tw = lib.twiss_from_mat6(lib.one_turn_matrix(ctx, lat, orbit, rf_on=False)[0], orbit)
    flip = [tw["phi_a"] / (2 * math.pi) < 0.5, tw["phi_b"] / (2 * math.pi) < 0.5, False]
    n_turn = 1024
    N = n_turn // 2
    q, st, _, _ = lib.fma(ctx, lat, np.array([[1e-6, 0, 1e-6, 0, 0, 0]]), n_turn)
    assert st[0] == 0
    for plane in range(3):
        want = (raw[plane] % 1.0) + 1.0 / N
        if flip[plane]:
            want = 1.0 - want
        for half in (0, 3):
            assert q[0, half + plane] == pytest.approx(want, abs=2e-5), plane


def test_fma_losses_reported(ctx, tmp_path):
    eles, p = rings.ring(20)
    lat = lib.Lattice(ctx, eles, p)
    off = np.array([[1e-3, 0, 1e-3, 0, 0, 0], [0.05, 0, 0, 0, 0, 0], [1e-3, 0, 0, 0, 0.3, 0]])
    q, st, tl, ie = lib.fma(ctx, lat, off, 128)
    assert list(st) == [0, 1, 2]     # alive; lost at the 20 mm aperture; z beyond lambda/4 = 0.15 m
    assert tl[1] == 1 and ie[1] >= 0
    path = str(tmp_path / "x.fm")
    lib.fma_write(path, off, q, st)
    lines = open(path).read().splitlines()
    assert len(lines) == 3            # header, the surviving particle, the '*' row
    assert lines[2].split()[3:] == ["*"] * 9
