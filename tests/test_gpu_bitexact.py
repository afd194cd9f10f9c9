"""GPU parity at the benchmark's sizes, bit for bit: the sm_100a tracker built with correctly
rounded transcendentals (libbmadgpu_cr.so) against the CPU oracle run with a correctly rounded
libm.

The device maps keep the reference's operation order (no FMA contraction); in that library they
call correctly rounded sin, cos, asin, atan2, sinh, cosh, exp and tan (csrc/crmath.cuh), and the element
invariants are packed with the same functions. The oracle -- the restatement of the reference's Fortran --
takes its libm functions from oracle_set_libm; installed with the same correctly rounded set
(checked against mpmath and against libquadmath on the CPU), it is the reference's algorithm
with a correctly rounded libm, and the GPU must reproduce it exactly: every coordinate, beta,
state, loss element, loss turn and location, after 1 and after 1000 turns, at 10,000 particles
on the 50-cell ring and 8,192 particles with losses on the 200-cell ring with multipoles and
edge fringes. (The default build, libbmadgpu.so, calls the device libm; it and glibc are
not correctly rounded -- glibc's sinh misrounds about a quarter of the ring's arguments -- and
test_gpu_parity.py holds it to the envelope that one-ulp libm differences produce.)"""
import importlib

import numpy as np
import pytest

from conftest import load_abi
from helpers import oracle_libm, oracle_track
from test_gpu_parity import _single_element_cases, gpu_track

pytestmark = pytest.mark.gpu
lib = importlib.import_module("bmad-ecosystem_b200.lib")
rings = importlib.import_module("bmad-ecosystem_b200.rings")
abi = load_abi()


@pytest.fixture(scope="module")
def cr_build():
    """libbmadgpu_cr.so for every object this module creates."""
    previous = lib.get_math()
    lib.set_math("cr")
    yield
    lib.set_math(previous)


@pytest.fixture(scope="module")
def ctx(cr_build):
    c = lib.Context(0)
    yield c
    c.close()


def test_the_correctly_rounded_build_is_loaded(ctx):
    assert lib.load()._name.endswith("libbmadgpu_cr.so")


def oracle_cr(eles, p, vec, n_turns, **kw):
    with oracle_libm("cr"):
        return oracle_track(eles, p, vec, n_turns, **kw)


def assert_identical(g, o, keys=("vec", "beta", "state", "ix_ele", "ix_turn", "location")):
    for k in keys:
        a, b = g[k], o[k]
        if a.dtype.kind == "f":
            na, nb = np.isnan(a), np.isnan(b)
            assert np.array_equal(na, nb), k
            a, b = a[~na], b[~nb]
            diff = np.flatnonzero(a.view(np.uint64) != b.view(np.uint64))
        else:
            diff = np.flatnonzero(a != b)
        assert diff.size == 0, "%s differs at %d places, first %s" % (k, diff.size, diff[:5])


@pytest.mark.parametrize("name", sorted(_single_element_cases()))
def test_single_element_bit_exact(ctx, name):
    eles = _single_element_cases()[name]
    p = abi.electron_param(3e9)
    rings.set_ref_time(eles, p)
    vec = rings.matched_gaussian(rings.ring(50)[0], 4096, seed=11, scale=3.0)
    assert_identical(gpu_track(ctx, eles, p, vec, 1), oracle_cr(eles, p, vec, 1))


def test_config0_full_size_bit_exact(ctx):
    """Config 0: the 50-cell ring, 10,000 particles of the matched Gaussian (seed 0), 1 and 1000
    turns."""
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 10000, seed=0)
    assert_identical(gpu_track(ctx, eles, p, vec, 1), oracle_cr(eles, p, vec, 1))
    t0 = np.zeros(vec.shape[1])
    g = gpu_track(ctx, eles, p, vec, 1000, t=t0)
    o = oracle_cr(eles, p, vec, 1000, t=t0)
    assert_identical(g, o)
    alive = o["state"] == abi.ALIVE
    # coord%t: FP64 on the device (from the turn's reference time), real(qp) in the reference
    assert np.max(np.abs(g["t"][alive] - o["t"][alive]) / np.abs(o["t"][alive])) < 1e-12


def test_config1_one_turn_bit_exact(ctx):
    eles, p = rings.ring(200, fringe=True, multipole_sigma=1e-4)
    vec = rings.matched_gaussian(eles, 4096, seed=3, scale=3.0)
    assert_identical(gpu_track(ctx, eles, p, vec, 1), oracle_cr(eles, p, vec, 1))


def test_config1_1000_turns_with_losses_bit_exact(ctx):
    """Config 1's ring (200 cells, b3..b10 sextupole multipoles, edge fringes), 8,192 particles of
    a Gaussian wide enough that some are lost at the aperture within the 1000 turns."""
    eles, p = rings.ring(200, fringe=True, multipole_sigma=1e-4)
    vec = rings.matched_gaussian(eles, 8192, seed=3, scale=14.0)
    g = gpu_track(ctx, eles, p, vec, 1000)
    o = oracle_cr(eles, p, vec, 1000)
    lost = o["state"] != abi.ALIVE
    assert lost.sum() >= 8 and (~lost).sum() > 4000, lost.sum()
    assert len(np.unique(o["ix_turn"][lost])) > 3       # losses spread over many turns
    assert_identical(g, o)


def test_losses_and_edge_inputs_bit_exact(ctx):
    """Heavy losses (a 12-sigma bunch) and the edge inputs of orbit_too_large and the apertures,
    NaN and infinite coordinates included."""
    from test_hostcheck_cpu import _edge_bunch
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 4096, seed=5, scale=12.0)
    g, o = gpu_track(ctx, eles, p, vec, 20), oracle_cr(eles, p, vec, 20)
    assert (o["state"] != abi.ALIVE).sum() > 100
    assert_identical(g, o)
    eles, p = rings.ring(20)
    vec = _edge_bunch()
    with np.errstate(invalid="ignore"):
        assert_identical(gpu_track(ctx, eles, p, vec, 2), oracle_cr(eles, p, vec, 2))


@pytest.mark.parametrize("case", ["orders_3_4_6_9", "skew_order", "octupole_b6"])
def test_multipole_kick_forms_bit_exact(ctx, case):
    eles, p = rings.ring(30)
    rng = np.random.default_rng(11)
    for e in eles:
        if e.key != abi.SEXTUPOLE:
            continue
        if case == "orders_3_4_6_9":
            for n in (3, 4, 6, 9):
                e.b_pole[n] = float(rng.normal(0, 1e-3))
        elif case == "skew_order":
            e.b_pole[4] = 2e-4
            e.a_pole[5] = -3e-4
        else:
            e.key = abi.OCTUPOLE
            e.k3 = 50.0
            e.k2 = 0.0
            e.b_pole[6] = 1e-3
    vec = rings.matched_gaussian(eles, 400, seed=5, scale=4.0)
    assert_identical(gpu_track(ctx, eles, p, vec, 5), oracle_cr(eles, p, vec, 5))


def test_perturbed_rings_bit_exact(ctx):
    """Misaligned and tilted quadrupoles and sextupoles with perturbed strengths (the batching and
    serving rings), 200 turns."""
    eles, p = rings.perturbed_ring(50, seed=1003)
    vec = rings.da_grid(2000)
    assert_identical(gpu_track(ctx, eles, p, vec, 200), oracle_cr(eles, p, vec, 200))


def test_batched_variants_bit_exact(ctx):
    """The batched path (several perturbed rings, uneven particle counts, one persistent launch per
    batch of turns) in the correctly rounded build: each variant bit-identical to the oracle."""
    lats, vecs, eles_p = [], [], []
    for v, n in enumerate((700, 2300, 1500)):
        eles, p = rings.perturbed_ring(50, seed=2000 + v)
        lats.append(lib.Lattice(ctx, eles, p))
        vecs.append(rings.da_grid(n))
        eles_p.append((eles, p))
    counts = [v.shape[1] for v in vecs]
    bunches = [lib.HostBunch.from_vec(v, p) for v, (_, p) in zip(vecs, eles_p)]
    whole = lib.concat_bunches(bunches)
    batch = lib.Batch(ctx, lats, counts)
    batch.upload(-1, whole)
    batch.track(64)
    out = lib.HostBunch(np.zeros((6, whole.n)), np.zeros(whole.n))
    batch.download(-1, out)
    parts = lib.split_bunch(out, counts)
    for (eles, p), vec, got in zip(eles_p, vecs, parts):
        o = oracle_cr(eles, p, vec, 64)
        g = dict(vec=got.vec, beta=got.beta, state=got.state, ix_ele=got.ix_ele, ix_turn=got.ix_turn,
                 location=got.location)
        lost = o["state"] != abi.ALIVE
        assert_identical(g, o, keys=("vec", "beta", "state"))
        assert np.array_equal(g["ix_ele"][lost], o["ix_ele"][lost])
        assert np.array_equal(g["ix_turn"][lost], o["ix_turn"][lost])
    batch.close()


def test_ring_with_rare_forms_bit_exact(ctx):
    """The full kernel instance over many turns: a ring with electric multipoles, full edge
    fringes, a rolled bend frame, a pitched sextupole, a collimator with phase-space windows and
    kickers, bit-identical to the oracle with a correctly rounded libm, losses included."""
    from test_hostcheck_cpu import _rare_ring
    eles, p = _rare_ring()
    vec = rings.matched_gaussian(rings.ring(20)[0], 4096, seed=17, scale=6.0)
    g, o = gpu_track(ctx, eles, p, vec, 100), oracle_cr(eles, p, vec, 100)
    assert (o["state"] != abi.ALIVE).sum() > 0
    assert_identical(g, o)
