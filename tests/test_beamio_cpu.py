"""Beam files (bmadgpu_beam_write_ascii / bmadgpu_beam_read_ascii), host-only, on CPU:
round trips in the reference's es23.15 layout (16 significant digits) and the exact layout (17
digits plus beta), lost particles with their state, element and location, alive-only output,
Fortran's three-digit exponent, and the reference's own ASCII::3 test beam
(regression_tests/hdf5_test/beam_1.dat, committed as tests/golden/hdf5_test_beam_1.dat)."""
import importlib
import os

import numpy as np
import pytest

lib = importlib.import_module("bmad-ecosystem_b200.lib")
abi = importlib.import_module("bmad-ecosystem_b200.abi")
rings = importlib.import_module("bmad-ecosystem_b200.rings")

REF_BEAM = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "hdf5_test_beam_1.dat")


def sample(n=300, seed=3):
    eles, p = rings.ring(10)
    b = lib.HostBunch.from_vec(rings.matched_gaussian(eles, n, seed=seed), p, t=np.random.default_rng(seed).normal(0, 1e-9, n))
    b.vec[0, 5] = 1.234567890123e-105        # three-digit exponent
    b.state[[3, 10, 11]] = [abi.LOST_POS_X, abi.LOST_NEG_Y, abi.LOST_PZ]
    b.ix_ele[[3, 10, 11]] = [17, 0, 35]
    b.location[:] = abi.DOWNSTREAM_END
    b.location[[3, 10, 11]] = [abi.DOWNSTREAM_END, abi.UPSTREAM_END, abi.INSIDE]
    return b, p


def test_exact_round_trip(tmp_path):
    b, p = sample()
    path = str(tmp_path / "beam.dat")
    lib.beam_write(path, b, p, flags=lib.BEAM_EXACT)
    r = lib.beam_read(path, p)
    for f in ("vec", "beta", "t", "state", "ix_ele", "location"):
        assert np.array_equal(getattr(r, f), getattr(b, f)), f


def test_reference_layout_round_trip(tmp_path):
    b, p = sample()
    path = str(tmp_path / "beam.dat")
    lib.beam_write(path, b, p)
    text = open(path).read().splitlines()
    assert text[0] == "# ix_bunch       =     1" and text[1].startswith("# n_particle     =")
    cols = [l for l in text if l.startswith("#!")][0].split()[1:]
    assert cols[:10] == ["index", "x", "px", "y", "py", "z", "pz", "p0c", "s_position", "time"]
    assert cols[-3:] == ["state", "ix_ele", "location"]
    assert "1.234567890123000-105" in open(path).read()          # Fortran's ES exponent form
    r = lib.beam_read(path, p)
    assert np.allclose(r.vec, b.vec, rtol=1e-15, atol=0)
    assert np.array_equal(r.state, b.state) and np.array_equal(r.location, b.location)
    # beta from pz as init_coord computes it (no beta column in the reference's layout)
    pc = p.p0c * (1 + r.vec[5])
    assert np.allclose(r.beta, pc / np.sqrt(pc * pc + p.mass ** 2), rtol=1e-15)


def test_alive_only(tmp_path):
    b, p = sample()
    path = str(tmp_path / "beam.dat")
    lib.beam_write(path, b, p, flags=lib.BEAM_ALIVE_ONLY)
    r = lib.beam_read(path, p)
    assert r.n == int(np.sum(b.state == abi.ALIVE))
    assert np.all(r.state == abi.ALIVE)


def test_reads_reference_ascii3_beam():
    p = abi.electron_param(3e9)
    r = lib.beam_read(REF_BEAM, p)
    assert r.n == 10
    # particle 7 of the file (the hdf5_test's first printed particle)
    assert np.allclose(r.vec[:, 6], [1.6387488057E-03, -2.9985054496E-06, 1.8144481648E-03, -7.8926417700E-05,
                                     -1.5942344121E-04, 5.2241291487E-04], rtol=0, atol=1e-20)
    assert list(r.state) == [1] * 10
    assert list(r.ix_ele[:3] + 1) == [7, 6, 5] and list(r.location[:3]) == [2, 4, 6]
