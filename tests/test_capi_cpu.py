"""C-ABI library checks that need no GPU: symbols, struct layout, host-side bookkeeping."""
import ctypes
import importlib
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_abi, load_oracle

lib = importlib.import_module("bmad-ecosystem_b200.lib")
rings = importlib.import_module("bmad-ecosystem_b200.rings")


@pytest.mark.parametrize("path", [lib.LIB_PATH, lib.LIB_CR_PATH], ids=["libbmadgpu", "libbmadgpu_cr"])
def test_library_exports_every_declared_symbol(path):
    """Both builds (device libm; correctly rounded transcendentals) export the whole C-ABI."""
    so = lib.load(path)
    declared = lib.declared_symbols()
    assert len(declared) >= 15
    missing = [s for s in declared if not hasattr(so, s)]
    assert not missing, missing
    out = subprocess.check_output(["nm", "-D", "--defined-only", path]).decode()
    for s in declared:
        assert (" T " + s) in out, s


@pytest.mark.parametrize("math", ["fast", "cr"])
def test_struct_layout_matches(math):
    previous = lib.get_math()
    lib.set_math(math)
    try:
        lib.check_layout()
        assert lib.load().bmadgpu_abi_version() == 1
    finally:
        lib.set_math(previous)


def test_ring_bookkeeping_matches_oracle():
    abi, orc = load_abi(), load_oracle()
    eles, param = rings.ring(50)
    steps, nbytes = lib.lattice_check(eles, param)
    assert 0 < nbytes < 64 * 1024   # identical cells pack into a small table
    for e, s in zip(eles, steps):
        n_or = orc.oracle_element_num_steps(ctypes.byref(e), ctypes.byref(param))
        if e.key in (abi.SEXTUPOLE, abi.RFCAVITY):
            assert s == n_or
        else:
            assert s == 1


def test_config1_ring_packs_and_sextupoles_use_one_step():
    eles, param = rings.ring(200, fringe=True, multipole_sigma=1e-4)
    steps, nbytes = lib.lattice_check(eles, param)
    assert nbytes < 200 * 1024
    abi = load_abi()
    assert all(s == 1 for e, s in zip(eles, steps) if e.key == abi.SEXTUPOLE)


@pytest.mark.parametrize("bad", ["elec_on_rfcavity", "bend_tilt", "bend_soft_edge", "abs_time"])
def test_unsupported_inputs_fail_loudly(bad):
    abi = load_abi()
    p = abi.electron_param(3e9)
    e = abi.default_element(abi.QUADRUPOLE, l=0.4, k1=0.5)
    if bad == "elec_on_rfcavity":
        e = abi.default_element(abi.RFCAVITY, l=0.4, voltage=1e6, rf_frequency=5e8)
        e.b_pole_elec[1] = 1e3
    elif bad == "bend_tilt":
        e = abi.default_element(abi.SBEND, l=1.0, g=0.01, tilt=1e-3)
    elif bad == "bend_soft_edge":
        e = abi.default_element(abi.SBEND, l=1.0, g=0.01, fringe_type=abi.FRINGE_SOFT_EDGE_ONLY)
    else:
        p.absolute_time_tracking = 1
    with pytest.raises(lib.BmadGpuError) as ei:
        lib.lattice_check([e], p)
    assert ei.value.code == abi.EUNSUPPORTED


def test_optics_of_benchmark_ring_is_stable():
    eles, _ = rings.ring(50)
    tw = rings.periodic_optics(eles)
    assert 0 < tw["tune_a"] < 1 and 0 < tw["tune_b"] < 1
    assert tw["beta_a"] > 0 and tw["beta_b"] > 0


def test_pitched_straight_elements_are_accepted():
    """Pitches and z_offset of straight elements are on the device path (the pitched offset form)."""
    abi = load_abi()
    p = abi.electron_param(3e9)
    for key in (abi.QUADRUPOLE, abi.SEXTUPOLE, abi.RFCAVITY):
        e = abi.default_element(key, l=0.4, k1=0.5, y_pitch=1e-3, x_pitch=-2e-3, z_offset=0.01)
        if key == abi.RFCAVITY:
            e.voltage, e.rf_frequency = 1e6, 5e8
        lib.lattice_check([e], p)


def test_misaligned_bends_and_electric_multipoles_are_accepted():
    """Offsets, pitches and z_offset of bends (the bend_shift frame) and electric multipoles of
    quadrupoles, sextupoles, octupoles, thick multipoles and bends are on the device path."""
    abi = load_abi()
    p = abi.electron_param(3e9)
    for kw in (dict(g=0.01, x_offset=1e-3), dict(g=0.01, y_pitch=1e-3, ref_tilt=0.1), dict(k1=0.3, z_offset=0.01),
               dict(g=0.01, roll=1e-3)):
        lib.lattice_check([abi.default_element(abi.SBEND, l=1.0, **kw)], p)
    for key in (abi.QUADRUPOLE, abi.SEXTUPOLE, abi.OCTUPOLE, abi.THICK_MULTIPOLE, abi.SBEND):
        e = abi.default_element(key, l=0.4, k1=0.5, g=0.01 if key == abi.SBEND else 0.0)
        e.b_pole_elec[1] = 1e3
        e.a_pole_elec[0] = -2e3
        lib.lattice_check([e], p)


def test_edge_fringes_are_accepted():
    """fringe_type full / hard_edge_only / soft_edge_only of quadrupoles and sextupoles and full of
    sbends (hard_multipole_edge_kick, soft_quadrupole_edge_kick, exact_bend_edge_kick)."""
    abi = load_abi()
    p = abi.electron_param(3e9)
    for ft in (abi.FRINGE_FULL, abi.FRINGE_HARD_EDGE_ONLY, abi.FRINGE_SOFT_EDGE_ONLY):
        for key in (abi.QUADRUPOLE, abi.SEXTUPOLE):
            lib.lattice_check([abi.default_element(key, l=0.4, k1=0.5, k2=3.0, fringe_type=ft, fq1=0.01)], p)
    lib.lattice_check([abi.default_element(abi.SBEND, l=1.0, g=0.01, e1=0.1, fint=0.5, hgap=0.02,
                                           fringe_type=abi.FRINGE_FULL)], p)



def test_collimators_and_kicked_monitors_are_accepted():
    """ecollimator / rcollimator (track_a_thick_multipole with phase-space windows) and monitors or
    instruments with hkick/vkick (has_hkick_attributes) are on the device path; scaled multipoles
    on an element without a reference strength are refused (convert_this_ab has no scale)."""
    abi = load_abi()
    p = abi.electron_param(3e9)
    lib.lattice_check([abi.default_element(abi.ECOLLIMATOR, l=0.5, x1_limit=1e-3, x2_limit=0.02, y1_limit=0.01,
                                           y2_limit=0.01, px_aperture_width2=1e-3, hkick=1e-5)], p)
    lib.lattice_check([abi.default_element(abi.RCOLLIMATOR, l=0.5, pz_aperture_width2=1e-3)], p)
    lib.lattice_check([abi.default_element(abi.MONITOR, l=0.2, hkick=1e-5, vkick=2e-5)], p)
    with pytest.raises(lib.BmadGpuError) as ei:
        lib.lattice_check([abi.default_element(abi.MONITOR, l=0.2, b_pole={2: 1e-3})], p)
    assert ei.value.code == abi.EUNSUPPORTED


def test_kickers_are_accepted():
    """hkicker / vkicker (kick) and kicker (hkick, vkick, scaled multipoles) are thick multipoles
    on the device path."""
    abi = load_abi()
    p = abi.electron_param(3e9)
    lib.lattice_check([abi.default_element(abi.HKICKER, l=0.2, kick=1e-4, tilt=0.1)], p)
    lib.lattice_check([abi.default_element(abi.VKICKER, l=0.2, kick=-1e-4)], p)
    lib.lattice_check([abi.default_element(abi.KICKER, l=0.2, hkick=1e-4, vkick=2e-4, b_pole={1: 2.0})], p)


def test_elseparators_are_accepted():
    """Elseparators (track_this_elsep with the longitudinal fringe) are on the device path."""
    abi = load_abi()
    p = abi.electron_param(3e9)
    lib.lattice_check([abi.default_element(abi.ELSEPARATOR, l=1.0, hkick=1e-5, vkick=2e-5, tilt=0.1)], p)
