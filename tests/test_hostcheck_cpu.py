"""The device element code compiled for the host (test-only build, csrc/hostcheck.cpp) against
the oracle: with the reference's operation order and no FMA contraction the two agree bit for
bit on the same libm, which pins the GPU algorithm before any GPU run."""
import ctypes
import importlib
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_abi
from helpers import oracle_libm, oracle_track

abi = load_abi()
rings = importlib.import_module("bmad-ecosystem_b200.rings")
# BMADGPU_HOSTCHECK_LIB / _CR_LIB: other builds of the same sources (the sanitizer test passes them)
HC = os.environ.get("BMADGPU_HOSTCHECK_LIB",
                    os.path.join(ROOT, "bmad-ecosystem_b200", "_build", "libbmadgpu_hostcheck.so"))
HC_CR = os.environ.get("BMADGPU_HOSTCHECK_CR_LIB",
                       os.path.join(ROOT, "bmad-ecosystem_b200", "_build", "libbmadgpu_hostcheck_cr.so"))


@pytest.fixture(scope="module")
def hc():
    if not os.path.exists(HC):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "bmad-ecosystem_b200", "csrc"), "hostcheck-lib"])
    return ctypes.CDLL(HC)


@pytest.fixture(scope="module")
def hc_cr():
    if not os.path.exists(HC_CR):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "bmad-ecosystem_b200", "csrc"), "hostcheck-lib"])
    lib = ctypes.CDLL(HC_CR)
    lib.bmadgpu_hostcheck_track = lib.bmadgpu_hostcheck_cr_track
    return lib


def host_track(hc, eles, p, vec, nt):
    arr = abi.element_array(eles)
    vec = np.ascontiguousarray(vec, dtype=np.float64).copy()
    n = vec.shape[1]
    pc = p.p0c * (1 + vec[5])
    beta = np.ascontiguousarray(np.where(vec[5] == 0, p.p0c / p.e_tot, pc / np.sqrt(pc * pc + p.mass ** 2)))
    st = np.ones(n, np.int32)
    ie = np.full(n, -1, np.int32)
    it = np.full(n, -1, np.int32)
    lo = np.zeros(n, np.int32)
    b = abi.Bunch(n, vec.ctypes.data, beta.ctypes.data, None, st.ctypes.data, ie.ctypes.data, it.ctypes.data,
                  lo.ctypes.data)
    assert hc.bmadgpu_hostcheck_track(arr, len(arr), ctypes.byref(p), ctypes.byref(b), nt) == 0
    return dict(vec=vec, beta=beta, state=st, ix_ele=ie, ix_turn=it, location=lo)


CASES = {
    "quad_misaligned": lambda E, ap: [E(abi.QUADRUPOLE, l=0.4, k1=-0.8, x_offset=3e-5, y_offset=-2e-5, tilt=1e-4, **ap)],
    "quad_multipoles": lambda E, ap: [E(abi.QUADRUPOLE, l=0.4, k1=0.8, b_pole={2: 1e-3, 3: -2e-4}, a_pole={2: 5e-4}, **ap)],
    "sextupole_b3_b10": lambda E, ap: [E(abi.SEXTUPOLE, l=0.2, k2=-18.0, b_pole={n: 1e-4 * (-1) ** n for n in range(3, 11)}, **ap)],
    "sextupole_steps": lambda E, ap: [E(abi.SEXTUPOLE, l=0.2, k2=12.0, x_offset=5e-5, tilt=-1e-4, num_steps=4, **ap)],
    "octupole": lambda E, ap: [E(abi.OCTUPOLE, l=0.3, k3=200.0, **ap)],
    "sbend_fringe": lambda E, ap: [E(abi.SBEND, l=1.5, g=2 * np.pi / 100 / 1.5, **ap)],
    "sbend_edges": lambda E, ap: [E(abi.SBEND, l=1.0, g=0.05, e1=0.03, e2=-0.02, fint=0.5, hgap=0.02, **ap)],
    "sbend_k1": lambda E, ap: [E(abi.SBEND, l=1.0, g=0.03, k1=0.2, **ap)],
    "sbend_multipoles": lambda E, ap: [E(abi.SBEND, l=1.0, g=0.03, b_pole={2: 1e-3}, fringe_type=abi.FRINGE_NONE, **ap)],
    "rf_thick": lambda E, ap: [E(abi.RFCAVITY, l=1.2, voltage=2e6, rf_frequency=500e6, phi0=0.05, **ap)],
    "multipole": lambda E, ap: [E(abi.MULTIPOLE, a_pole={0: 1e-4, 1: 0.02, 2: 0.5}, b_pole={1: 0.1, 2: 0.2}, x_offset=1e-4)],
    "ab_multipole": lambda E, ap: [E(abi.AB_MULTIPOLE, a_pole={2: 0.3}, b_pole={1: 0.01, 2: 0.5}, tilt=0.1)],
    "sextupole_pitched": lambda E, ap: [E(abi.SEXTUPOLE, l=0.6, k2=1.0, tilt=0.52, num_steps=10, x_offset=0.05,
                                          y_pitch=0.001, z_offset=0.02, **ap)],
    "quad_pitched": lambda E, ap: [E(abi.QUADRUPOLE, l=0.4, k1=-0.8, x_pitch=-2e-3, y_pitch=1e-3, z_offset=-0.01,
                                     y_offset=1e-4, **ap)],
    "rf_pitched": lambda E, ap: [E(abi.RFCAVITY, l=1.2, voltage=2e6, rf_frequency=500e6, x_pitch=1e-3, tilt=0.1,
                                   x_offset=1e-4, **ap)],
    # electric multipoles (kicks with the energy change, the longitudinal fringe at the edges)
    "quad_elec": lambda E, ap: [E(abi.QUADRUPOLE, l=0.4, k1=0.8, b_pole_elec={0: 2e5, 1: 3e6}, a_pole_elec={2: 1e6},
                                  r0_elec=0.05, x_offset=2e-4, tilt=0.05, **ap)],
    "quad_elec_exit_edge_only": lambda E, ap: [E(abi.QUADRUPOLE, l=0.4, k1=-0.8, b_pole_elec={1: 3e6, 3: 4e7},
                                                 fringe_at=abi.EXIT_END, **ap)],
    "sextupole_elec": lambda E, ap: [E(abi.SEXTUPOLE, l=0.3, k2=10.0, a_pole_elec={0: -1e5, 2: 5e6}, num_steps=3,
                                       y_pitch=1e-3, **ap)],
    "sbend_elec": lambda E, ap: [E(abi.SBEND, l=1.0, g=0.03, e1=0.02, b_pole={2: 1e-3}, b_pole_elec={0: -2e5},
                                   a_pole_elec={1: 2e6}, r0_elec=3.0, **ap)],
    # misaligned bends: the bend_shift frame (g or ref_tilt non-zero) and the straight form
    "sbend_offsets": lambda E, ap: [E(abi.SBEND, l=1.0, g=0.03, x_offset=1e-3, y_offset=-5e-4, x_pitch=2e-4,
                                      y_pitch=-1e-4, z_offset=0.01, **ap)],
    "sbend_ref_tilt_offsets": lambda E, ap: [E(abi.SBEND, l=0.8, g=0.05, e1=0.02, e2=-0.01, ref_tilt=0.3,
                                               x_offset=1e-3, y_pitch=2e-4, **ap)],
    "sbend_g0_offsets": lambda E, ap: [E(abi.SBEND, l=0.6, k1=0.2, x_offset=1e-3, y_pitch=1e-3, z_offset=-0.02, **ap)],
    "sbend_roll": lambda E, ap: [E(abi.SBEND, l=1.0, g=0.03, roll=0.02, x_offset=1e-3, y_pitch=2e-4, **ap)],
    "sbend_roll_ref_tilt": lambda E, ap: [E(abi.SBEND, l=1.0, g=0.03, e1=0.02, roll=-0.01, ref_tilt=0.2, **ap)],
    "sbend_g0_ref_tilt": lambda E, ap: [E(abi.SBEND, l=0.6, k1=0.3, k2=3.0, ref_tilt=0.1, x_offset=2e-3,
                                          y_pitch=1e-3, num_steps=10, **ap)],
    # collimators: phase-space windows before the x/y limits, asymmetric elliptical limits
    "ecollimator_windows": lambda E, ap: [E(abi.ECOLLIMATOR, l=0.5, x1_limit=1e-3, x2_limit=0.02, y1_limit=0.01,
                                            y2_limit=0.008, px_aperture_width2=4e-4, px_aperture_center=1e-5,
                                            py_aperture_width2=3e-4, pz_aperture_width2=2e-3, hkick=1e-5,
                                            x_offset=1e-4, tilt=0.05)],
    "rcollimator_windows": lambda E, ap: [E(abi.RCOLLIMATOR, l=0.5, x1_limit=0.02, x2_limit=0.02, y1_limit=0.01,
                                            y2_limit=0.01, px_aperture_width2=3e-4, py_aperture_width2=2e-4,
                                            py_aperture_center=-1e-5, z_aperture_width2=5e-3, pz_aperture_width2=1.5e-3,
                                            vkick=-1e-5)],
    "monitor_kicks": lambda E, ap: [E(abi.MONITOR, l=0.2, hkick=2e-5, vkick=-1e-5, x_offset=1e-4, **ap)],
    "elseparator_h": lambda E, ap: [E(abi.ELSEPARATOR, l=1.0, hkick=2e-5, num_steps=5, x_offset=1e-4, tilt=0.1, **ap)],
    "elseparator_hv": lambda E, ap: [E(abi.ELSEPARATOR, l=1.0, hkick=-1e-5, vkick=2e-5, num_steps=3, y_pitch=1e-4,
                                       **ap)],
    "hkicker": lambda E, ap: [E(abi.HKICKER, l=0.3, kick=3e-5, num_steps=4, x_offset=1e-4, tilt=0.1, **ap)],
    "vkicker": lambda E, ap: [E(abi.VKICKER, l=0.3, kick=-2e-5, y_pitch=1e-4, **ap)],
    "kicker_multipole": lambda E, ap: [E(abi.KICKER, l=0.3, hkick=1e-5, vkick=2e-5, b_pole={0: 0.2, 1: 3.0},
                                         num_steps=3, tilt=-0.05, **ap)],
    "elliptical_asymmetric": lambda E, ap: [E(abi.DRIFT, l=1.0, aperture_type=abi.APERTURE_ELLIPTICAL, x1_limit=0.004,
                                              x2_limit=0.006, y1_limit=0.002, y2_limit=0.003)],
    # higher-order edge fringes: hard-edge multipole, soft quadrupole edge, exact bend edge
    "quad_fringe_full": lambda E, ap: [E(abi.QUADRUPOLE, l=0.4, k1=0.8, fringe_type=abi.FRINGE_FULL, fq1=0.02, fq2=-0.01,
                                         tilt=0.3, **ap)],
    "quad_hard_edge_exit": lambda E, ap: [E(abi.QUADRUPOLE, l=0.4, k1=-0.8, fringe_type=abi.FRINGE_HARD_EDGE_ONLY,
                                            fringe_at=abi.EXIT_END, b_pole_elec={1: 3e6}, **ap)],
    "quad_soft_edge": lambda E, ap: [E(abi.QUADRUPOLE, l=0.4, k1=0.8, fringe_type=abi.FRINGE_SOFT_EDGE_ONLY, fq1=0.05,
                                       fq2=0.01, **ap)],
    "sextupole_fringe_full": lambda E, ap: [E(abi.SEXTUPOLE, l=0.3, k2=20.0, fringe_type=abi.FRINGE_FULL,
                                              x_offset=1e-3, **ap)],
    "octupole_fringe_full": lambda E, ap: [E(abi.OCTUPOLE, l=0.3, k3=200.0, fringe_type=abi.FRINGE_FULL, **ap)],
    "sbend_fringe_full": lambda E, ap: [E(abi.SBEND, l=1.0, g=0.05, k1=0.2, e1=0.1, e2=-0.05, fint=0.5, hgap=0.03,
                                          fringe_type=abi.FRINGE_FULL, **ap)],
    "sbend5_like": lambda E, ap: [E(abi.SBEND, l=0.6, g=0.01, e1=0.1, e2=0.2, num_steps=10, fringe_type=abi.FRINGE_FULL,
                                    x_offset=0.002, y_pitch=0.001, ref_tilt=0.1, fint=0.7, hgap=2.0,
                                    a_pole={0: 0.001, 1: 10.0, 3: 100.0}, b_pole_elec={0: -2e5}, a_pole_elec={1: 2e6}, **ap)],
    "sbend7_like": lambda E, ap: [E(abi.SBEND, l=0.6, g=0.01, e1=0.1, e2=0.2, num_steps=10, x_offset=0.002,
                                    y_pitch=0.001, ref_tilt=0.1, a_pole={0: 0.01, 1: 0.1}, vkick=-1e-4,
                                    b_pole_elec={0: -2e5}, a_pole_elec={1: 2e6}, r0_mag=2.0, r0_elec=3.0, **ap)],
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_device_code_on_host_is_bit_exact(hc, name):
    ap = dict(x1_limit=0.02, x2_limit=0.02, y1_limit=0.01, y2_limit=0.01)
    eles = CASES[name](abi.default_element, ap)
    p = abi.electron_param(3e9)
    rings.set_ref_time(eles, p)
    vec = rings.matched_gaussian(rings.ring(50)[0], 1000, seed=11, scale=3.0)
    o = oracle_track(eles, p, vec, 1)
    h = host_track(hc, eles, p, vec, 1)
    for k in ("vec", "beta", "state"):
        assert np.array_equal(h[k], o[k]), k


def test_config1_ring_bit_exact_on_host(hc):
    eles, p = rings.ring(200, fringe=True, multipole_sigma=1e-4)
    vec = rings.matched_gaussian(eles, 200, seed=3, scale=3.0)
    o = oracle_track(eles, p, vec, 5)
    h = host_track(hc, eles, p, vec, 5)
    assert np.array_equal(h["vec"], o["vec"])
    assert np.array_equal(h["state"], o["state"])


def test_losses_on_host_match_oracle(hc):
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 1500, seed=5, scale=12.0)
    o = oracle_track(eles, p, vec, 10)
    h = host_track(hc, eles, p, vec, 10)
    lost = o["state"] != abi.ALIVE
    assert lost.sum() > 50
    for k in ("state", "ix_ele", "ix_turn", "location"):
        assert np.array_equal(h[k][lost] if k != "state" else h[k], o[k][lost] if k != "state" else o[k]), k


def test_noise_envelope_is_ulp_scale_after_one_turn():
    """The 1-ulp libm perturbation used as the GPU's long-term yardstick stays at the 1e-12 level
    after one turn (it is a rounding-level perturbation, not a modelling change)."""
    from helpers import noise_track, per_particle_err
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 300, seed=0)
    o = oracle_track(eles, p, vec, 1)
    z = noise_track(eles, p, vec, 1)
    e = per_particle_err(z["vec"], o["vec"])
    assert 0 < e.max() < 2e-11


@pytest.mark.parametrize("case", ["zero_middle_orders", "skew_order", "octupole_b6"])
def test_multipole_kick_forms_bit_exact_on_host(hc, case):
    """Sextupoles and octupoles whose kicks take the branch-free normal-multipole form (every a_n
    zero, b_0 = b_1 = 0), with exactly zero orders in the middle of the range, and one with a skew
    order (the general form) stay bit-identical to the oracle over several turns."""
    eles, p = rings.ring(30)
    rng = np.random.default_rng(7)
    for e in eles:
        if e.key != abi.SEXTUPOLE:
            continue
        if case == "zero_middle_orders":
            poles = {n: float(rng.normal(0, 1e-3)) for n in (3, 4, 6, 9)}   # b5, b7, b8 exactly zero
            for n, v in poles.items():
                e.b_pole[n] = v
        elif case == "skew_order":
            e.b_pole[4] = 2e-4
            e.a_pole[5] = -3e-4
        else:
            e.key = abi.OCTUPOLE
            e.k3 = 50.0
            e.k2 = 0.0
            e.b_pole[6] = 1e-3
    vec = rings.matched_gaussian(eles, 300, seed=2, scale=6.0)
    o = oracle_track(eles, p, vec, 4)
    h = host_track(hc, eles, p, vec, 4)
    alive = o["state"] == abi.ALIVE
    assert 0 < alive.sum() < 300           # some losses, some survivors
    assert np.array_equal(h["vec"][:, alive], o["vec"][:, alive])
    for k in ("state", "ix_ele", "ix_turn"):
        assert np.array_equal(h[k], o[k]), k


def test_rf_phase_fold_outside_the_bucket_bit_exact_on_host(hc):
    """Particles beyond half an RF wavelength: the reference folds the RF time with modulo2 in
    real(qp) (particle_rf_time.f90:115), where t - k 2 amp is exact; the device carries the folded
    time in double-double and must give the same pz bits as the oracle's __float128 path."""
    cav = rings.rf_cavity()
    drift = abi.default_element(abi.DRIFT, l=0.5)
    eles = rings.set_ref_time([cav, drift, cav], rings.ring(1)[1])
    p = rings.ring(1)[1]
    rng = np.random.default_rng(3)
    n = 4000
    vec = np.zeros((6, n))
    vec[4] = rng.uniform(-0.9, 0.9, n)          # half wavelength at 500 MHz: 0.30 m
    vec[5] = rng.normal(0, 1e-3, n)
    o = oracle_track(eles, p, vec, 2)
    h = host_track(hc, eles, p, vec, 2)
    assert np.sum(np.abs(vec[4]) > 0.3) > n // 2
    for k in ("vec", "beta", "state"):
        assert np.array_equal(h[k], o[k]), k


def _edge_bunch():
    """Particles at the edges of orbit_too_large and the apertures: beyond max_aperture_limit in
    either plane, 1 + pz < 0, px^2 + py^2 > (1 + pz)^2, just inside and just outside the 20 mm /
    10 mm apertures, and NaN or infinite coordinates (which every comparison lets through, as in
    the reference)."""
    rows = [
        [2e3, 0, 0, 0, 0, 0], [-2e3, 0, 0, 0, 0, 0], [0, 0, 2e3, 0, 0, 0], [0, 0, -2e3, 0, 0, 0],
        [0, 0, 0, 0, 0, -1.5], [0, 1.2, 0, 0, 0, 0], [0, 0.1, 0, -1.3, 0, 0.0],
        [0.0199999, 0, 0, 0, 0, 0], [0.0200001, 0, 0, 0, 0, 0], [0, 0, -0.0100001, 0, 0, 0],
        [np.nan, 0, 0, 0, 0, 0], [0, np.nan, 0, 0, 0, 0], [0, 0, 0, 0, np.nan, 0], [0, 0, 0, 0, 0, np.nan],
        [np.inf, 0, 0, 0, 0, 0], [0, 0, 0, 0, 0, 0], [1e-3, 1e-4, -1e-3, 2e-5, 1e-3, 1e-3],
    ]
    return np.ascontiguousarray(np.array(rows, dtype=np.float64).T)


def test_edge_inputs_on_host_match_oracle(hc):
    eles, p = rings.ring(20)
    vec = _edge_bunch()
    with np.errstate(invalid="ignore"):
        o = oracle_track(eles, p, vec, 2)
        h = host_track(hc, eles, p, vec, 2)
    for k in ("state", "ix_ele", "ix_turn", "location"):
        assert np.array_equal(h[k], o[k]), (k, h[k], o[k])
    assert np.array_equal(h["vec"], o["vec"], equal_nan=True)
    lost = o["state"] != abi.ALIVE
    assert lost[[0, 1, 2, 3, 4, 5, 6, 8, 9]].all()
    assert o["state"][0] == abi.LOST_POS_X and o["state"][1] == abi.LOST_NEG_X
    assert o["state"][2] == abi.LOST_POS_Y and o["state"][3] == abi.LOST_NEG_Y
    assert o["state"][4] == abi.LOST_PZ


# ---- correctly rounded transcendentals: the device's arithmetic on the CPU --------------------

@pytest.mark.parametrize("name", sorted(CASES))
def test_device_code_with_cr_libm_is_bit_exact(hc_cr, name):
    """The host build of the device maps with the correctly rounded functions (maps and element
    invariants, as in the product library) against the oracle with the same functions installed."""
    ap = dict(x1_limit=0.02, x2_limit=0.02, y1_limit=0.01, y2_limit=0.01)
    eles = CASES[name](abi.default_element, ap)
    p = abi.electron_param(3e9)
    rings.set_ref_time(eles, p)
    vec = rings.matched_gaussian(rings.ring(50)[0], 1000, seed=11, scale=3.0)
    with oracle_libm("cr"):
        o = oracle_track(eles, p, vec, 1)
    h = host_track(hc_cr, eles, p, vec, 1)
    for k in ("vec", "beta", "state"):
        assert np.array_equal(h[k], o[k]), k


def test_config1_ring_with_cr_libm_bit_exact(hc_cr):
    eles, p = rings.ring(200, fringe=True, multipole_sigma=1e-4)
    vec = rings.matched_gaussian(eles, 200, seed=3, scale=3.0)
    with oracle_libm("cr"):
        o = oracle_track(eles, p, vec, 5)
    h = host_track(hc_cr, eles, p, vec, 5)
    assert np.array_equal(h["vec"], o["vec"])
    assert np.array_equal(h["state"], o["state"])


def test_cr_libm_equals_an_independent_correctly_rounded_libm():
    """The oracle tracking the 50-cell ring with the device's correctly rounded functions and with
    libquadmath's rounded once: the same bits, so the device's functions are correctly rounded on
    the arguments tracking produces, not only on the random ones of test_crmath_cpu.py."""
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 64, seed=4, scale=3.0)
    with oracle_libm("cr"):
        a = oracle_track(eles, p, vec, 20)
    with oracle_libm("quad"):
        b = oracle_track(eles, p, vec, 20)
    assert np.array_equal(a["vec"], b["vec"])
    assert np.array_equal(a["state"], b["state"])
    with oracle_libm("cr"):
        pass
    c = oracle_track(eles, p, vec, 20)        # the host's libm again: not correctly rounded
    assert not np.array_equal(a["vec"], c["vec"])


def _rare_ring():
    """A 20-cell ring carrying every rare element form at once: a quadrupole with electric
    multipoles, a full (hard and soft) edge fringe and fq1/fq2, a rolled and offset bend with
    fringe_type full, a pitched sextupole, an ecollimator with phase-space windows, kickers."""
    E = abi.default_element
    eles, p = rings.ring(20)
    quads = [i for i, e in enumerate(eles) if e.key == abi.QUADRUPOLE]
    bends = [i for i, e in enumerate(eles) if e.key == abi.SBEND]
    sexts = [i for i, e in enumerate(eles) if e.key == abi.SEXTUPOLE]
    q = eles[quads[3]]
    q.b_pole_elec[1] = 2e5
    q.a_pole_elec[2] = 1e6
    q.fringe_type = abi.FRINGE_FULL
    q.fq1, q.fq2 = 0.01, -0.005
    b = eles[bends[5]]
    b.x_offset, b.roll, b.y_pitch = 2e-4, 1e-3, 1e-4
    b.fringe_type, b.e1, b.fint, b.hgap = abi.FRINGE_FULL, 0.01, 0.5, 0.02
    b.fintx, b.hgapx = b.fint, b.hgap
    eles[sexts[4]].z_offset = 1e-3
    eles[sexts[4]].x_pitch = 2e-4
    extra = [E(abi.ECOLLIMATOR, l=0.1, x1_limit=0.015, x2_limit=0.015, y1_limit=0.008, y2_limit=0.008,
               px_aperture_width2=2e-3, py_aperture_width2=1.5e-3),
             E(abi.HKICKER, l=0.1, kick=1e-6), E(abi.KICKER, l=0.1, hkick=-1e-6, vkick=5e-7)]
    eles = eles[:10] + extra + eles[10:]
    rings.set_ref_time(eles, p)
    return eles, p


def test_ring_with_rare_forms_on_host(hc, hc_cr):
    """Many turns of a ring with every rare form (the full kernel's path), bit-identical to the
    oracle with glibc and with the correctly rounded libm, losses included."""
    eles, p = _rare_ring()
    vec = rings.matched_gaussian(rings.ring(20)[0], 400, seed=17, scale=6.0)
    o = oracle_track(eles, p, vec, 30)
    h = host_track(hc, eles, p, vec, 30)
    for k in ("vec", "beta", "state", "ix_ele", "ix_turn"):
        assert np.array_equal(h[k], o[k]), k
    assert (o["state"] != abi.ALIVE).sum() > 0 and (o["state"] == abi.ALIVE).sum() > 100
    with oracle_libm("cr"):
        o = oracle_track(eles, p, vec, 30)
    h = host_track(hc_cr, eles, p, vec, 30)
    for k in ("vec", "beta", "state", "ix_ele", "ix_turn"):
        assert np.array_equal(h[k], o[k]), k


def test_edge_inputs_through_rare_forms_on_host(hc):
    """The edge inputs (beyond the aperture limits, NaN and infinite coordinates) through the ring
    with every rare element form: the host build of the device code equals the oracle."""
    eles, p = _rare_ring()
    vec = _edge_bunch()
    with np.errstate(invalid="ignore"):
        o = oracle_track(eles, p, vec, 2)
        h = host_track(hc, eles, p, vec, 2)
    for k in ("vec", "beta", "state", "ix_ele", "ix_turn"):
        a, b = h[k], o[k]
        if a.dtype.kind == "f":
            assert np.array_equal(np.isnan(a), np.isnan(b)), k
            a, b = a[~np.isnan(a)], b[~np.isnan(b)]
        assert np.array_equal(a, b), k
