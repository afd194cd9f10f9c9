"""GPU parity: the sm_100a tracker (through the C-ABI) against the CPU oracle and the golden
vectors.

Errors are relative to the coordinate's RMS over the bunch (a coordinate near zero has no
relative error of its own). The device code compiled for the host is bit-identical to the oracle
(tests/test_hostcheck_cpu.py); on the GPU the only difference left is the device libm (sin, cos,
asin, atan2, sinh, cosh), about one ulp from glibc's. Hence:
  - one element: <= 1e-12;
  - one turn of a ring: <= 1e-11 (1-ulp libm noise alone reaches ~5e-12 after one turn of the
    100-bend ring: each exact-bend step forms x from terms ~1e3 times larger);
  - many turns: the GPU's spread from the oracle must stay within a small factor of the spread
    that 1-ulp libm perturbations alone cause (helpers.noise_track) -- the nonlinear dynamics
    amplify any ulp difference, so a fixed 1e-9 after 1000 turns is met by the median particle
    only up to that amplification;
  - losses: same particles, same element, same turn, same state code."""
import ctypes
import importlib
import json
import os

import numpy as np
import pytest

from conftest import ROOT, load_abi
from helpers import coord_floor, noise_track, oracle_track, per_particle_err, rel_err

pytestmark = pytest.mark.gpu
lib = importlib.import_module("bmad-ecosystem_b200.lib")
rings = importlib.import_module("bmad-ecosystem_b200.rings")
abi = load_abi()


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    yield c
    c.close()


def gpu_track(ctx, elements, param, vec, n_turns, moments=False, t=None, **tuning):
    saved = ctx.get_tuning()
    if tuning:
        ctx.set_tuning(**tuning)
    lat = lib.Lattice(ctx, elements, param)
    b = lib.HostBunch.from_vec(vec, param, t=t)
    mom = lib.track_bunch(ctx, lat, b, n_turns=n_turns, moments=moments)
    if tuning:
        ctx.set_tuning(**saved)
    return dict(vec=b.vec, beta=b.beta, state=b.state, ix_ele=b.ix_ele, ix_turn=b.ix_turn, location=b.location,
                t=b.t, moments=mom)


def assert_close(g, o, tol, floor_frac=1.0, alive_only=True):
    mask = (o["state"] == abi.ALIVE) & (g["state"] == abi.ALIVE) if alive_only else slice(None)
    fl = coord_floor(o["vec"][:, mask]) if np.any(mask) else 1.0
    err = rel_err(g["vec"][:, mask], o["vec"][:, mask], fl)
    assert err.size == 0 or err.max() <= tol, "max rel err %g" % err.max()
    return err.max() if err.size else 0.0


# ---- golden vectors through the device path ----------------------------------------------------

# Golden cases whose element form the device path refuses (BMADGPU_EUNSUPPORTED), by name, with
# the reason; every other case runs on the GPU against its golden line. None is refused: the
# electric multipoles of QUADRUPOLE1-3 and SBEND3/5/7, the misaligned-bend frame of the bends
# and SBEND5's exact edge (fringe_type full) are on the device.
REFUSED_ON_DEVICE = {}


def _golden_cases():
    data = json.load(open(os.path.join(ROOT, "tests", "golden", "tracking_method_bmad_standard.json")))
    return [(c, data) for c in data["cases"]]


def _golden_id(c):
    return c["name"] if isinstance(c, dict) and "name" in c else ""


@pytest.mark.parametrize("case,data", _golden_cases(), ids=_golden_id)
def test_golden_vectors_on_gpu(ctx, case, data):
    p = abi.electron_param(data["e_tot"], charge=data["charge"])
    e = abi.default_element(getattr(abi, case["key"]), **case["attrs"])
    if case["name"] in REFUSED_ON_DEVICE:
        with pytest.raises(lib.BmadGpuError) as ex:
            lib.lattice_check([e], p)
        assert ex.value.code == abi.EUNSUPPORTED
        return
    vec = np.array(data["start"], dtype=np.float64).reshape(6, 1)
    g = gpu_track(ctx, [e], p, vec, 1)
    assert g["state"][0] == abi.ALIVE
    for i in range(6):
        want = case["expected_vec"][i]
        assert abs(g["vec"][i, 0] - want) <= case["tol"] + 5e-11 * abs(want), (case["name"], i)


def _m6_cases():
    data = json.load(open(os.path.join(ROOT, "tests", "golden", "mat6_calc_method_tracking.json")))
    return [(c, data) for c in data["cases"]]


@pytest.mark.parametrize("case,data", _m6_cases(), ids=_golden_id)
def test_mat6_by_tracking_on_gpu(ctx, case, data):
    """Transfer matrix and vec0 of each element by central differences of GPU tracking (thirteen
    particles, as make_mat6_tracking forms them) against the reference's mat6_calc_method_test
    "Tracking" lines, ABS 1e-9."""
    from test_oracle_golden import M6_NOT_RESTATED, matrix_by_tracking
    p = abi.electron_param(data["e_tot"], charge=data["charge"])
    e = abi.default_element(getattr(abi, case["key"]), **case["attrs"])
    if case["name"] in M6_NOT_RESTATED:
        with pytest.raises(lib.BmadGpuError) as ex:
            lib.lattice_check([e], p)
        assert ex.value.code == abi.EUNSUPPORTED
        return

    def track(starts):
        g = gpu_track(ctx, [e], p, np.array(starts, dtype=np.float64).T.copy(), 1)
        return list(g["vec"].T), list(g["state"])

    mat, vec0 = matrix_by_tracking(track, data["start"], data["d_orb"])
    want = np.asarray(case["expected_mat6"])
    assert np.all(np.abs(mat - want) <= np.asarray(case["tol_rows"])[:, None] + 5e-14 * np.abs(want)), (case["name"], mat - want)
    want0 = np.asarray(case["expected_vec0"])
    assert np.all(np.abs(vec0 - want0) <= case["tol_vec0"] + 5e-14 * np.abs(want0)), (case["name"], vec0 - want0)


def _ap_cases():
    return json.load(open(os.path.join(ROOT, "tests", "golden", "aperture_test_collimators.json")))["cases"]


@pytest.mark.parametrize("case", _ap_cases(), ids=lambda c: c["name"])
def test_aperture_test_collimators_on_gpu(ctx, case):
    """The reference's zero-length ecollimator / rcollimator (aperture checked at the exit) tracked on
    the GPU from each aperture_test grid point: the loss states of its S lines."""
    p = abi.electron_param(3.1e9, charge=1.0)
    e = abi.default_element(getattr(abi, case["key"]), **case["attrs"])
    vec = np.array(case["vecs"], dtype=np.float64).T.copy()
    g = gpu_track(ctx, [e], p, vec, 1)
    assert list(g["state"]) == case["expected_state"], (case["name"], list(g["state"]))


# ---- single elements of every kind against the oracle -----------------------------------------

def _single_element_cases():
    ap = dict(x1_limit=0.02, x2_limit=0.02, y1_limit=0.01, y2_limit=0.01)
    E = abi.default_element
    return {
        "drift": [E(abi.DRIFT, l=2.5, **ap)],
        "quad_f": [E(abi.QUADRUPOLE, l=0.4, k1=0.8, **ap)],
        "quad_d_misaligned": [E(abi.QUADRUPOLE, l=0.4, k1=-0.8, x_offset=3e-5, y_offset=-2e-5, tilt=1e-4, **ap)],
        "quad_multipoles": [E(abi.QUADRUPOLE, l=0.4, k1=0.8, b_pole={2: 1e-3, 3: -2e-4}, a_pole={2: 5e-4}, **ap)],
        "sextupole": [E(abi.SEXTUPOLE, l=0.2, k2=12.0, **ap)],
        "sextupole_b3_b10": [E(abi.SEXTUPOLE, l=0.2, k2=-18.0, b_pole={n: 1e-4 * (-1) ** n for n in range(3, 11)}, **ap)],
        "sextupole_misaligned": [E(abi.SEXTUPOLE, l=0.2, k2=12.0, x_offset=5e-5, tilt=-1e-4, num_steps=4, **ap)],
        "octupole": [E(abi.OCTUPOLE, l=0.3, k3=200.0, **ap)],
        "sbend": [E(abi.SBEND, l=1.5, g=2 * np.pi / 100 / 1.5, fringe_type=abi.FRINGE_NONE, **ap)],
        "sbend_fringe": [E(abi.SBEND, l=1.5, g=2 * np.pi / 100 / 1.5, **ap)],
        "sbend_edges_fint": [E(abi.SBEND, l=1.0, g=0.05, e1=0.03, e2=-0.02, fint=0.5, hgap=0.02, **ap)],
        "sbend_k1": [E(abi.SBEND, l=1.0, g=0.03, k1=0.2, **ap)],
        "sbend_multipoles": [E(abi.SBEND, l=1.0, g=0.03, b_pole={2: 1e-3}, fringe_type=abi.FRINGE_NONE, **ap)],
        "rf_thin": [E(abi.RFCAVITY, l=0.0, voltage=2e6, rf_frequency=500e6, **ap)],
        "rf_thick": [E(abi.RFCAVITY, l=1.2, voltage=2e6, rf_frequency=500e6, phi0=0.05, **ap)],
        "multipole": [E(abi.MULTIPOLE, a_pole={0: 1e-4, 1: 0.02, 2: 0.5}, b_pole={1: 0.1, 2: 0.2}, x_offset=1e-4)],
        "ab_multipole": [E(abi.AB_MULTIPOLE, a_pole={2: 0.3}, b_pole={1: 0.01, 2: 0.5}, tilt=0.1)],
        "marker": [E(abi.MARKER)],
        "sextupole_pitched": [E(abi.SEXTUPOLE, l=0.6, k2=1.0, tilt=0.52, num_steps=10, x_offset=0.05, y_pitch=0.001,
                                z_offset=0.02, **ap)],
        "quad_pitched": [E(abi.QUADRUPOLE, l=0.4, k1=-0.8, x_pitch=-2e-3, y_pitch=1e-3, z_offset=-0.01, y_offset=1e-4,
                           **ap)],
        "rf_pitched": [E(abi.RFCAVITY, l=1.2, voltage=2e6, rf_frequency=500e6, x_pitch=1e-3, tilt=0.1, x_offset=1e-4,
                         **ap)],
        "quad_elec": [E(abi.QUADRUPOLE, l=0.4, k1=0.8, b_pole_elec={0: 2e5, 1: 3e6}, a_pole_elec={2: 1e6}, r0_elec=0.05,
                        x_offset=2e-4, tilt=0.05, **ap)],
        "quad_elec_exit_edge_only": [E(abi.QUADRUPOLE, l=0.4, k1=-0.8, b_pole_elec={1: 3e6, 3: 4e7},
                                       fringe_at=abi.EXIT_END, **ap)],
        "sextupole_elec": [E(abi.SEXTUPOLE, l=0.3, k2=10.0, a_pole_elec={0: -1e5, 2: 5e6}, num_steps=3, y_pitch=1e-3,
                             **ap)],
        "sbend_elec": [E(abi.SBEND, l=1.0, g=0.03, e1=0.02, b_pole={2: 1e-3}, b_pole_elec={0: -2e5}, a_pole_elec={1: 2e6},
                         r0_elec=3.0, **ap)],
        "sbend_offsets": [E(abi.SBEND, l=1.0, g=0.03, x_offset=1e-3, y_offset=-5e-4, x_pitch=2e-4, y_pitch=-1e-4,
                            z_offset=0.01, **ap)],
        "sbend_ref_tilt_offsets": [E(abi.SBEND, l=0.8, g=0.05, e1=0.02, e2=-0.01, ref_tilt=0.3, x_offset=1e-3,
                                     y_pitch=2e-4, **ap)],
        "sbend_g0_offsets": [E(abi.SBEND, l=0.6, k1=0.2, x_offset=1e-3, y_pitch=1e-3, z_offset=-0.02, **ap)],
        "sbend_roll": [E(abi.SBEND, l=1.0, g=0.03, roll=0.02, x_offset=1e-3, y_pitch=2e-4, **ap)],
        "sbend_roll_ref_tilt": [E(abi.SBEND, l=1.0, g=0.03, e1=0.02, roll=-0.01, ref_tilt=0.2, **ap)],
        "quad_fringe_full": [E(abi.QUADRUPOLE, l=0.4, k1=0.8, fringe_type=abi.FRINGE_FULL, fq1=0.02, fq2=-0.01, tilt=0.3,
                               **ap)],
        "quad_soft_edge": [E(abi.QUADRUPOLE, l=0.4, k1=0.8, fringe_type=abi.FRINGE_SOFT_EDGE_ONLY, fq1=0.05, fq2=0.01,
                             **ap)],
        "sextupole_fringe_full": [E(abi.SEXTUPOLE, l=0.3, k2=20.0, fringe_type=abi.FRINGE_FULL, x_offset=1e-3, **ap)],
        "sbend_fringe_full": [E(abi.SBEND, l=1.0, g=0.05, k1=0.2, e1=0.1, e2=-0.05, fint=0.5, hgap=0.03,
                                fringe_type=abi.FRINGE_FULL, **ap)],
        "sbend5_like": [E(abi.SBEND, l=0.6, g=0.01, e1=0.1, e2=0.2, num_steps=10, fringe_type=abi.FRINGE_FULL,
                          x_offset=0.002, y_pitch=0.001, ref_tilt=0.1, fint=0.7, hgap=2.0,
                          a_pole={0: 0.001, 1: 10.0, 3: 100.0}, b_pole_elec={0: -2e5}, a_pole_elec={1: 2e6}, **ap)],
        "ecollimator_windows": [E(abi.ECOLLIMATOR, l=0.5, x1_limit=1e-3, x2_limit=0.02, y1_limit=0.01, y2_limit=0.008,
                                  px_aperture_width2=4e-4, px_aperture_center=1e-5, py_aperture_width2=3e-4,
                                  pz_aperture_width2=2e-3, hkick=1e-5, x_offset=1e-4, tilt=0.05)],
        "rcollimator_windows": [E(abi.RCOLLIMATOR, l=0.5, x1_limit=0.02, x2_limit=0.02, y1_limit=0.01, y2_limit=0.01,
                                  px_aperture_width2=3e-4, py_aperture_width2=2e-4, py_aperture_center=-1e-5,
                                  z_aperture_width2=5e-3, pz_aperture_width2=1.5e-3, vkick=-1e-5)],
        "monitor_kicks": [E(abi.MONITOR, l=0.2, hkick=2e-5, vkick=-1e-5, x_offset=1e-4, **ap)],
        "elseparator_hv": [E(abi.ELSEPARATOR, l=1.0, hkick=-1e-5, vkick=2e-5, num_steps=3, y_pitch=1e-4, **ap)],
        "hkicker": [E(abi.HKICKER, l=0.3, kick=3e-5, num_steps=4, x_offset=1e-4, tilt=0.1, **ap)],
        "kicker_multipole": [E(abi.KICKER, l=0.3, hkick=1e-5, vkick=2e-5, b_pole={0: 0.2, 1: 3.0}, num_steps=3,
                               tilt=-0.05, **ap)],
        "elliptical_asymmetric": [E(abi.DRIFT, l=1.0, aperture_type=abi.APERTURE_ELLIPTICAL, x1_limit=0.004, x2_limit=0.006,
                                    y1_limit=0.002, y2_limit=0.003)],
        "sbend7_like": [E(abi.SBEND, l=0.6, g=0.01, e1=0.1, e2=0.2, num_steps=10, x_offset=0.002, y_pitch=0.001,
                          ref_tilt=0.1, a_pole={0: 0.01, 1: 0.1}, vkick=-1e-4, b_pole_elec={0: -2e5},
                          a_pole_elec={1: 2e6}, r0_mag=2.0, r0_elec=3.0, **ap)],
    }


@pytest.mark.parametrize("name", sorted(_single_element_cases()))
def test_single_element_matches_oracle(ctx, name):
    eles = _single_element_cases()[name]
    p = abi.electron_param(3e9)
    rings.set_ref_time(eles, p)
    vec = rings.matched_gaussian(rings.ring(50)[0], 4096, seed=11, scale=3.0)
    o = oracle_track(eles, p, vec, 1)
    g = gpu_track(ctx, eles, p, vec, 1)
    assert np.array_equal(g["state"], o["state"])
    assert_close(g, o, 1e-12)
    lost = o["state"] != abi.ALIVE
    assert np.array_equal(g["ix_ele"][lost], o["ix_ele"][lost])
    assert np.array_equal(g["location"][lost], o["location"][lost])


# ---- rings -------------------------------------------------------------------------------------

def test_config0_ring_one_turn(ctx):
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 2000, seed=0)
    t0 = np.zeros(vec.shape[1])
    o = oracle_track(eles, p, vec, 1, t=t0)
    g = gpu_track(ctx, eles, p, vec, 1, t=t0)
    assert np.array_equal(g["state"], o["state"])
    assert_close(g, o, 1e-11)
    assert np.max(np.abs(g["beta"] - o["beta"]) / o["beta"]) < 1e-14
    alive = o["state"] == abi.ALIVE
    assert np.max(np.abs(g["t"][alive] - o["t"][alive]) / np.abs(o["t"][alive])) < 1e-12


def _envelope_check(g, o, z, factor):
    alive = (o["state"] == abi.ALIVE) & (g["state"] == abi.ALIVE) & (z["state"] == abi.ALIVE)
    eg = per_particle_err(g["vec"][:, alive], o["vec"][:, alive])
    ez = per_particle_err(z["vec"][:, alive], o["vec"][:, alive])
    for q in (0.5, 0.9, 0.99):
        assert np.quantile(eg, q) <= factor * np.quantile(ez, q), (q, np.quantile(eg, q), np.quantile(ez, q))
    assert eg.max() <= factor * ez.max(), (eg.max(), ez.max())
    return eg, ez


def test_config0_ring_1000_turns(ctx):
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 256, seed=0)
    o = oracle_track(eles, p, vec, 1000)
    g = gpu_track(ctx, eles, p, vec, 1000)
    z = noise_track(eles, p, vec, 1000)
    assert np.array_equal(g["state"], o["state"])
    eg, ez = _envelope_check(g, o, z, 4.0)
    assert np.median(eg) < 2e-8


def test_config1_ring_with_multipoles_and_fringe(ctx):
    eles, p = rings.ring(200, fringe=True, multipole_sigma=1e-4)
    vec = rings.matched_gaussian(eles, 512, seed=3, scale=3.0)
    o = oracle_track(eles, p, vec, 1)
    g = gpu_track(ctx, eles, p, vec, 1)
    assert np.array_equal(g["state"], o["state"])
    assert_close(g, o, 1e-11)
    o = oracle_track(eles, p, vec, 50)
    g = gpu_track(ctx, eles, p, vec, 50)
    z = noise_track(eles, p, vec, 50)
    assert np.array_equal(g["state"], o["state"])
    _envelope_check(g, o, z, 4.0)


def test_losses_match_oracle(ctx):
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 4096, seed=5, scale=12.0)
    o = oracle_track(eles, p, vec, 20)
    g = gpu_track(ctx, eles, p, vec, 20)
    z = noise_track(eles, p, vec, 20)
    lost = o["state"] != abi.ALIVE
    assert lost.sum() > 100
    assert np.array_equal(g["state"], o["state"])
    assert np.array_equal(g["ix_ele"][lost], o["ix_ele"][lost])
    assert np.array_equal(g["ix_turn"][lost], o["ix_turn"][lost])
    assert np.array_equal(g["location"][lost], o["location"][lost])
    _envelope_check(g, o, z, 4.0)


def test_moments_match_oracle(ctx):
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 3000, seed=7, scale=8.0)
    o = oracle_track(eles, p, vec, 10, moments=True)
    g = gpu_track(ctx, eles, p, vec, 10, moments=True)
    assert np.array_equal(g["moments"][:, 0], o["moments"][:, 0])
    scale = np.maximum(np.abs(o["moments"]), 1e-30)
    assert np.max(np.abs(g["moments"] - o["moments"]) / scale) < 1e-9


@pytest.mark.parametrize("tuning", [dict(block=64), dict(block=256), dict(stage_smem=0),
                                    dict(turns_per_launch=7, compact=1), dict(turns_per_launch=3, compact=0)])
def test_launch_shapes_agree(ctx, tuning):
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 3000, seed=9, scale=10.0)
    base = gpu_track(ctx, eles, p, vec, 25)
    alt = gpu_track(ctx, eles, p, vec, 25, **tuning)
    for k in ("vec", "beta", "state", "ix_ele", "ix_turn", "location"):
        assert np.array_equal(base[k], alt[k]), k


@pytest.mark.parametrize("variant", [dict(block=128, ctas_per_sm=6), dict(block=256, ctas_per_sm=0),
                                     dict(block=64, ctas_per_sm=12), dict(block=512, ctas_per_sm=0)])
def test_register_budget_variants_are_bitwise_identical(ctx, variant):
    eles, p = rings.ring(200, fringe=True, multipole_sigma=1e-4)
    vec = rings.matched_gaussian(eles, 2000, seed=4, scale=4.0)
    base = gpu_track(ctx, eles, p, vec, 3)
    alt = gpu_track(ctx, eles, p, vec, 3, **variant)
    for k in ("vec", "beta", "state"):
        assert np.array_equal(base[k], alt[k]), k


def test_autotuner_leaves_bunch_untouched(ctx):
    import torch
    eles, p = rings.ring(50)
    lat = lib.Lattice(ctx, eles, p)
    hb = lib.HostBunch.from_vec(rings.matched_gaussian(eles, 50000, seed=1), p)
    d = {k: torch.from_numpy(getattr(hb, k)).cuda() for k in ("vec", "beta", "state")}
    torch.cuda.synchronize()
    v = abi.Bunch(hb.n, d["vec"].data_ptr(), d["beta"].data_ptr(), None, d["state"].data_ptr(), None, None, None)
    chosen = lib.autotune(ctx, lat, v)
    assert chosen["block"] in (64, 128, 256, 512)
    assert np.array_equal(d["vec"].cpu().numpy(), hb.vec)
    assert np.array_equal(d["state"].cpu().numpy(), hb.state)
    ctx.set_tuning(block=128, ctas_per_sm=0, stage_smem=1, turns_per_launch=0, compact=0)


@pytest.mark.parametrize("case", ["orders_3_4_6_9", "skew_order", "octupole_b6", "orders_to_5"])
def test_multipole_kick_forms_match_oracle(ctx, case):
    """The device's kick forms on orders the benchmark rings do not reach: the branch-free normal
    form for 4 to 10 orders (with exactly zero orders inside the range), an octupole, and a skew
    order (the general form), each against the oracle after one and five turns."""
    eles, p = rings.ring(30)
    rng = np.random.default_rng(11)
    for e in eles:
        if e.key != abi.SEXTUPOLE:
            continue
        if case == "orders_3_4_6_9":
            for n in (3, 4, 6, 9):
                e.b_pole[n] = float(rng.normal(0, 1e-3))
        elif case == "orders_to_5":
            for n in (3, 5):
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
    for nt in (1, 5):
        o = oracle_track(eles, p, vec, nt)
        g = gpu_track(ctx, eles, p, vec, nt)
        assert np.array_equal(g["state"], o["state"])
        assert_close(g, o, 1e-11 if nt == 1 else 1e-9)


def test_edge_inputs_match_oracle(ctx):
    """Particles at the edges of orbit_too_large and the apertures, and NaN or infinite coordinates
    (alive in the reference, whose comparisons let NaN through): states, loss elements, turns and
    locations equal the oracle's; coordinates agree, NaN where the oracle has NaN."""
    from test_hostcheck_cpu import _edge_bunch
    eles, p = rings.ring(20)
    vec = _edge_bunch()
    with np.errstate(invalid="ignore"):
        o = oracle_track(eles, p, vec, 2)
        g = gpu_track(ctx, eles, p, vec, 2)
    for k in ("state", "ix_ele", "ix_turn", "location"):
        assert np.array_equal(g[k], o[k]), (k, g[k], o[k])
    assert np.array_equal(np.isnan(g["vec"]), np.isnan(o["vec"]))
    fin = np.isfinite(o["vec"]) & np.isfinite(g["vec"])
    scale = np.maximum(np.abs(o["vec"]), 1e-12)
    with np.errstate(invalid="ignore"):
        diff = np.abs(g["vec"] - o["vec"])
    assert np.all(diff[fin] <= 1e-11 * scale[fin])
