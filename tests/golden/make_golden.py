"""Generates the golden-vector fixtures in this folder from the reference's own regression tests.

Run in a checkout that has the reference at REF (default /root/reference); the outputs are small
JSON files committed next to this script, so nothing at test time reads the reference.

Sources (paths inside bmad-sim/bmad-ecosystem):
  regression_tests/tracking_method_test/tracking_method_test.bmad   element definitions, start orbit
  regression_tests/tracking_method_test/output.correct              "NAME: Bmad_Standard" lines
  regression_tests/fringe_test/fringe_test.bmad, output.correct     hwang_bend_edge_kick goldens
  regression_tests/mat6_calc_method_test/mat6_calc_method_test.bmad, output.correct
                                                                    transfer matrices by tracking
  regression_tests/aperture_test/aperture_test.bmad, .f90, output.correct
                                                                    collimator aperture states
  regression_tests/coord_test/coord_test.bmad, .f90, output.correct offset_particle of bends

Element attributes are transcribed below from the .bmad lines cited beside each entry; Bmad's
parser defaults are applied explicitly (tilt flag -> pi/4 quad, pi/6 sextupole, pi/8 octupole,
parser_set_attribute_mod.f90:1813-1823; multipole tN flag -> pi/(2N+2), :1809).
"""
import json
import math
import os
import re
import sys

REF = os.environ.get("BMAD_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))
PI = 3.141592653589793238462643383279

# particle_start, tracking_method_test.bmad:9-14; l1[e_tot] = 1e6, :141. The file sets no
# parameter[particle], so the species is Bmad's default positron (bmad_parser.f90:966): charge +1.
TM_START = [0.001, 0.002, 0.003, 0.004, 0.005, 0.006]
TM_E_TOT = 1e6
TM_CHARGE = 1.0

_sb0 = dict(a_pole={0: 0.01, 1: 0.1}, vkick=-0.0001, b_pole_elec={0: -2e3}, a_pole_elec={1: 2e4}, r0_mag=2.0,
            r0_elec=3.0)  # :79
def rbend_to_sbend(attrs):
    """The parser's rbend conversion (bmad_parser_mod.f90:5186-5225, fiducial_pt none): the given
    l is the chord; the arc length follows from g, the angle is g l, e1 and e2 each gain half the
    angle, and the element is an sbend from then on."""
    import math
    a = dict(attrs)
    l_chord, g = a.pop("l"), a.get("g", 0.0)
    if g != 0:
        ang = 2.0 * math.asin(0.5 * l_chord * g)
        l = l_chord * ang / (2.0 * math.sin(0.5 * ang))
    else:
        l = l_chord
    angle = g * l
    a["l"] = l
    a["e1"] = a.get("e1", 0.0) + 0.5 * angle
    a["e2"] = a.get("e2", 0.0) + 0.5 * angle
    if angle != 0:
        a["g"] = angle / l
    return a


_rb0 = dict(a_pole={0: 0.01, 1: 0.1}, vkick=-0.0001, b_pole_elec={0: -2e3}, a_pole_elec={1: 2e4}, r0_mag=2.0,
            r0_elec=3.0)  # :80
_q0 = dict(a_pole={0: 0.01, 1: 0.1}, vkick=-0.0001, b_pole_elec={0: -2e3}, a_pole_elec={1: 2e4})  # :62

TM_ELEMENTS = {
    # name: (key, attributes, source line in tracking_method_test.bmad)
    "DRIFT1": ("DRIFT", dict(l=4.5, num_steps=10, x_offset=0.05, y_pitch=0.001, tilt=0.1), 27),
    "INSTRUMENT1": ("INSTRUMENT", dict(l=4.5, num_steps=10), 41),
    "HKICKER1": ("HKICKER", dict(l=4.5, kick=0.005, num_steps=10, x_offset=0.05, y_pitch=0.001, tilt=0.1), 40),
    "ELSEPARATOR1": ("ELSEPARATOR", dict(l=4.5, hkick=0.005, num_steps=10, x_offset=0.05, y_pitch=0.001, tilt=0.1), 30),
    "ELSEPARATOR2": ("ELSEPARATOR", dict(l=4.5, vkick=0.005, num_steps=10, x_offset=0.05, y_pitch=0.001, tilt=0.1), 31),
    "VKICKER1": ("VKICKER", dict(l=4.5, kick=0.005, num_steps=10, x_offset=0.05, y_pitch=0.001, tilt=0.1), 124),
    "KICKER1": ("KICKER", dict(l=4.5, b_pole={0: 0.002}, vkick=0.003, num_steps=10, x_offset=0.05, y_pitch=0.001,
                               tilt=0.1), 42),
    "ECOLLIMATOR1": ("ECOLLIMATOR", dict(l=4.5, x1_limit=0.2, x2_limit=0.2, y1_limit=0.1, y2_limit=0.1, num_steps=10,
                                         x_offset=0.02, y_pitch=0.001, tilt=0.1, hkick=0.01, vkick=0.002), 29),
    "RCOLLIMATOR1": ("RCOLLIMATOR", dict(l=4.5, x1_limit=0.2, x2_limit=0.2, y1_limit=0.1, y2_limit=0.1, num_steps=10,
                                         x_offset=0.02, y_pitch=0.001, tilt=0.1), 68),
    "MONITOR1": ("MONITOR", dict(l=4.5, num_steps=10), 55),
    "MULTIPOLE1": ("MULTIPOLE", dict(a_pole={1: 1.0, 3: 4.5}, b_pole={1: PI / (2 * 1 + 2), 3: 0.31 * PI},
                                     x_offset=0.05), 56),
    "AB_MULTIPOLE1": ("AB_MULTIPOLE", dict(a_pole={2: 1e2}, b_pole={2: 1e2}, x_offset=0.02, tilt=0.1), 20),
    "OCTUPOLE1": ("OCTUPOLE", dict(l=4.5, k3=1e3, tilt=PI / 8.0, num_steps=10, x_offset=0.01,
                                   y_pitch=0.001), 58),
    "SEXTUPOLE1": ("SEXTUPOLE", dict(l=0.6, k2=1.0, tilt=PI / 6.0, num_steps=10, x_offset=0.05,
                                     y_pitch=0.001), 93),
    "RFCAVITY1": ("RFCAVITY", dict(l=4.5, rf_frequency=500e6, voltage=1e5, phi0=0.1, num_steps=10,
                                   x_offset=0.05, y_pitch=0.001, tilt=0.1), 69),
    "RFCAVITY3": ("RFCAVITY", dict(rf_frequency=500e6, voltage=1e5, phi0=0.1, num_steps=10, x_offset=0.05,
                                   y_pitch=0.001, tilt=0.1, a_pole={2: 0.02}), 73),
    "QUADRUPOLE1": ("QUADRUPOLE", dict(_q0, l=0.6, k1=1.0, tilt=PI / 4.0, num_steps=10, x_offset=0.05,
                                       y_pitch=0.001), 63),
    "QUADRUPOLE2": ("QUADRUPOLE", dict(_q0, l=0.6, k1=-1.0, tilt=PI / 4.0, num_steps=10, x_offset=0.05,
                                       y_pitch=0.001), 64),
    "QUADRUPOLE3": ("QUADRUPOLE", dict(_q0, l=0.6, k1=1e-20, tilt=PI / 4.0, num_steps=10, x_offset=0.05,
                                       y_pitch=0.001), 65),
    # fringe_type full: hard_multipole_edge_kick at both edges (soft edge without fq1/fq2)
    "QUADRUPOLE4": ("QUADRUPOLE", dict(_q0, l=0.6, k1=1.0, tilt=PI / 4.0, num_steps=10, x_offset=0.05,
                                       y_pitch=0.001, fringe_type=4), 66),
    "QUADRUPOLE5": ("QUADRUPOLE", dict(_q0, l=0.6, k1=-1.0, tilt=PI / 4.0, num_steps=10, x_offset=0.05,
                                       y_pitch=0.001, fringe_type=4), 67),
    "THICK_MULTIPOLE1": ("THICK_MULTIPOLE", dict(l=4.5, a_pole={2: 1.0}, b_pole={3: 20.0}, x_offset=0.02, tilt=0.1),
                         123),
    # sb0 (:79) with the pieces of sbend3 (:84) and sbend7 (:91): offsets, pitch and ref_tilt on a
    # bend (the bend_shift frame of offset_particle), magnetic and electric multipoles
    "SBEND3": ("SBEND", dict(_sb0, l=0.6, k1=0.3, k2=3.0, num_steps=10, x_offset=0.05, y_pitch=0.001,
                             ref_tilt=0.1), 84),
    "SBEND7": ("SBEND", dict(_sb0, l=0.6, g=0.01, e1=0.1, e2=0.2, num_steps=10, x_offset=0.05, y_pitch=0.001,
                             ref_tilt=0.1), 91),
    # rbends (l = the chord), converted as the parser converts them
    "RBEND4": ("SBEND", rbend_to_sbend(dict(_rb0, l=0.6, g=0.01, dg=-0.0099, e1=0.1, e2=0.2, num_steps=10,
                                            fringe_type=4, x_offset=0.05, y_pitch=0.001, ref_tilt=0.1)), 85),
    "RBEND6": ("SBEND", rbend_to_sbend(dict(_rb0, l=0.6, g=0.01, dg=-0.0099999, e1=0.1, e2=0.2, num_steps=10,
                                            x_offset=0.05, y_pitch=0.001, ref_tilt=0.1)), 89),
    # fringe_type full: exact_bend_edge_kick with fint = 0.7, hgap = 2 (:87-88)
    "SBEND5": ("SBEND", dict(_sb0, l=0.6, g=0.01, e1=0.1, e2=0.2, num_steps=10, fringe_type=4, x_offset=0.05,
                             y_pitch=0.001, ref_tilt=0.1, fint=0.7, hgap=2.0), 87),
}

# mat6_calc_method_test.bmad: e_tot 1e6, default species (positron), the same particle_start as
# tracking_method_test (:9-14). The "Tracking" lines hold the transfer matrix that
# make_mat6_tracking (bmad/low_level/make_mat6_tracking.f90:26-110) forms by central differences
# of bmad_standard tracking with steps bmad_com%d_orb = 1e-5 (bmad_struct.f90:2315), and
# vec0 = end orbit - matrix * start orbit. Elements on the path, with their .bmad lines:
_m_q0 = dict(a_pole={0: 0.01, 1: 0.1}, vkick=-0.0001, b_pole_elec={0: -2e3}, a_pole_elec={1: 2e5})  # :64
_m_sb0 = dict(a_pole={0: 0.001, 1: 0.1}, vkick=-0.0001, b_pole_elec={0: -2e3}, a_pole_elec={1: 2e3})  # :80
FULL = 4  # fringe_type full$ (bmad_struct.f90:168)
_m_mis = dict(num_steps=10, x_offset=0.05, y_pitch=0.001)
_m_rb0 = dict(a_pole={0: 0.001, 1: 0.1}, vkick=-0.0001, b_pole_elec={0: -2e3}, a_pole_elec={1: 2e3})  # :81
M6_ELEMENTS = {
    "AB_MULTIPOLE1": ("AB_MULTIPOLE", dict(a_pole={2: 1e3}, b_pole={2: 1e3}, x_offset=0.02, tilt=0.1), 19),
    "DRIFT1": ("DRIFT", dict(l=4.5, tilt=0.1, **_m_mis), 23),
    "INSTRUMENT1": ("INSTRUMENT", dict(l=4.5, num_steps=10), 34),
    "HKICKER1": ("HKICKER", dict(l=4.5, kick=0.005, tilt=0.1, **_m_mis), 33),
    "ELSEPARATOR1": ("ELSEPARATOR", dict(l=4.5, hkick=0.005, tilt=0.1, **_m_mis), 26),
    "ELSEPARATOR2": ("ELSEPARATOR", dict(l=4.5, vkick=0.005, tilt=0.1, **_m_mis), 27),
    "VKICKER1": ("VKICKER", dict(l=4.5, kick=0.005, tilt=0.1, **_m_mis), 125),
    "KICKER1": ("KICKER", dict(l=4.5, hkick=0.003, vkick=0.003, tilt=0.1, **_m_mis), 35),
    "ECOLLIMATOR1": ("ECOLLIMATOR", dict(l=4.5, x1_limit=0.2, x2_limit=0.2, y1_limit=0.1, y2_limit=0.1, num_steps=10,
                                         x_offset=0.02, y_pitch=0.001, tilt=0.1, hkick=0.01, vkick=0.002), 25),
    "RCOLLIMATOR1": ("RCOLLIMATOR", dict(l=4.5, x1_limit=0.2, x2_limit=0.2, y1_limit=0.1, y2_limit=0.1, num_steps=10,
                                         x_offset=0.02, y_pitch=0.001, tilt=0.1), 71),
    "MONITOR1": ("MONITOR", dict(l=4.5, num_steps=10), 56),
    "MULTIPOLE1": ("MULTIPOLE", dict(a_pole={1: 1.0, 3: 4.5}, b_pole={1: PI / (2 * 1 + 2), 3: 0.31 * PI},
                                     x_offset=0.05), 57),
    "OCTUPOLE1": ("OCTUPOLE", dict(l=4.5, k3=1e3, tilt=PI / 8.0, num_steps=10, x_offset=0.01, y_pitch=0.001), 59),
    "QUADRUPOLE1": ("QUADRUPOLE", dict(_m_q0, l=0.6, k1=1.0, tilt=0.1, **_m_mis), 65),
    "QUADRUPOLE2": ("QUADRUPOLE", dict(_m_q0, l=0.6, k1=-1.0, tilt=PI / 4.0, **_m_mis), 66),
    "QUADRUPOLE3": ("QUADRUPOLE", dict(_m_q0, l=0.6, k1=1e-20, tilt=PI / 4.0, **_m_mis), 67),
    "QUADRUPOLE4": ("QUADRUPOLE", dict(_m_q0, l=0.6, k1=1.0, tilt=PI / 4.0, fringe_type=FULL, **_m_mis), 68),
    "QUADRUPOLE5": ("QUADRUPOLE", dict(_m_q0, l=0.6, k1=-1.0, tilt=PI / 4.0, fringe_type=FULL, **_m_mis), 69),
    "RFCAVITY1": ("RFCAVITY", dict(l=4.5, rf_frequency=500e6, voltage=5e5, phi0=0.1, tilt=0.1, b_pole={2: 0.002},
                                   **_m_mis), 72),
    "SBEND3": ("SBEND", dict(_m_sb0, l=0.6, k1=0.3, k2=3.0, ref_tilt=0.1, **_m_mis), 84),
    "SBEND5": ("SBEND", dict(_m_sb0, l=0.6, g=0.01, e1=0.1, e2=0.2, fringe_type=FULL, ref_tilt=0.1,
                             a_pole={0: 0.001, 1: 10.0, 3: 100.0}, fint=0.7, hgap=2.0, **_m_mis), 87),
    "SBEND7": ("SBEND", dict(_m_sb0, l=0.6, g=0.01, e1=0.1, e2=0.2, ref_tilt=0.1, a_pole={0: 0.001, 1: 10.0, 3: 100.0},
                             **_m_mis), 91),
    "SEXTUPOLE1": ("SEXTUPOLE", dict(l=0.6, k2=1.0, tilt=PI / 6.0, **_m_mis), 94),
    "RBEND4": ("SBEND", rbend_to_sbend(dict(_m_rb0, l=0.6, g=0.01, dg=-0.009999, e1=0.1, e2=0.2, fringe_type=FULL,
                                            ref_tilt=0.1, b_pole={1: 10.0, 3: 100.0}, **_m_mis)), 85),
    "RBEND6": ("SBEND", rbend_to_sbend(dict(_m_rb0, l=0.6, g=0.01, dg=-0.009999999, e1=0.1, e2=0.2, ref_tilt=0.1,
                                            **_m_mis)), 89),
    "THICK_MULTIPOLE1": ("THICK_MULTIPOLE", dict(l=4.5, a_pole={2: 1.0}, b_pole={2: 20.0}, x_offset=0.02, tilt=0.1),
                         124),
}

# aperture_test.bmad:23-35 (ec, rc) and check_this_aperture (aperture_test.f90:116-220), which
# calls check_aperture_limit at second_track_edge on 9-point grids around each window's edges
# and prints the states (S lines) and param%unstable_factor (U lines, 3 digits). The driver's
# grid constants (xw2 = 0.01, x0, eps = 1e-5, ...) are default-kind REAL literals, i.e. single
# precision widened to double; that rounding shows in the printed unstable factors (9.98E-06 in
# RC_U_zPz+), so the grid is built here with the same float32 values.
_win = dict(px_aperture_width2=0.01, px_aperture_center=0.01, py_aperture_width2=0.015, z_aperture_width2=0.2,
            z_aperture_center=-0.6, pz_aperture_width2=0.03, pz_aperture_center=0.02, x1_limit=1e-10,
            x2_limit=0.02, y1_limit=0.015, y2_limit=0.015)
AP_ELEMENTS = {"EC": ("ECOLLIMATOR", _win, 23), "RC": ("RCOLLIMATOR", _win, 30)}


def aperture_grids():
    """The six grids of check_this_aperture: name -> 9 phase-space vectors (i outer, j inner)."""
    import numpy as np
    f = lambda v: float(np.float32(v))
    out = {}
    for sign, tag in ((-1, "-"), (1, "+")):
        xw2, x0, yw2, y0, eps = f(0.01), f(0.01), f(0.015), 0.0, f(1e-5)
        g = []
        for i in (-1, 0, 1):
            for j in (-1, 0, 1):
                g.append([0.0, x0 + i * (xw2 + sign * eps), 0.0, y0 + j * (yw2 + sign * eps), -0.6, 0.02])
        out["Pxy" + tag] = g
        g = []
        for i in (-1, 0, 1):
            for j in (-1, 0, 1):
                g.append([x0 + i * (xw2 + sign * eps), 0.1 if sign < 0 else 0.0, y0 + j * (yw2 + sign * eps), 0.0,
                          -0.6, 0.02])
        out["xy" + tag] = g
        xw2, x0, yw2, y0 = f(0.2), f(-0.6), f(0.03), f(0.02)
        g = []
        for i in (-1, 0, 1):
            for j in (-1, 0, 1):
                g.append([0.0, 0.01, 0.0, 0.0, x0 + i * (xw2 + sign * eps), y0 + j * (yw2 + sign * eps)])
        out["zPz" + tag] = g
    return out

# coord_test.bmad:38-40 (line l2: e_tot 1e8 electrons): b0, b1 (offsets, pitches, roll) and b2
# (the same with ref_tilt = 2), and offset_track_drift (coord_test.f90:124-160) at orientation 1,
# direction 1: offset_particle set ("Drift-In"), track1 through the element with its offsets,
# pitches, roll and ref_tilt zeroed (zero_ele_offsets.f90:14-54, "Drift-Xfer"), offset_particle
# unset ("Drift-Out").
CT_ELEMENTS = {
    "B0": ("SBEND", dict(l=2.0, g=0.1, dg=-0.1), 38),
    "B1": ("SBEND", dict(l=2.0, g=0.1, dg=-0.1, x_offset=0.2, y_offset=0.3, x_pitch=0.1, y_pitch=0.2, roll=0.3), 39),
    "B2": ("SBEND", dict(l=2.0, g=0.1, dg=-0.1, x_offset=0.2, y_offset=0.3, x_pitch=0.1, y_pitch=0.2, roll=0.3,
                         ref_tilt=2.0), 40),
}

# fringe_test.bmad: e_tot 1e6 electrons, particle_start, b: sbend ...
FR_START = [0.01, 0.02, 0.03, 0.04, 0.00, 0.5]
FR_ELEMENT = dict(e1=0.1, e2=-0.2, k1=0.1, g=0.1, fint=0.5, hgap=0.4)


def parse_output_correct(path):
    out = {}
    for ln, line in enumerate(open(path), start=1):
        m = re.match(r'\s*"([^"]+)"\s+(ABS|REL|VEC_REL)\s+(\S+)\s+(.*)$', line)
        if not m:
            continue
        vals = [float(v) for v in m.group(4).split()]
        out[m.group(1)] = dict(tol_type=m.group(2), tol=float(m.group(3)), values=vals, line=ln)
    return out


def main():
    tm = parse_output_correct(os.path.join(REF, "regression_tests/tracking_method_test/output.correct"))
    cases = []
    for name, (key, attrs, src_line) in TM_ELEMENTS.items():
        g = tm[name + ": Bmad_Standard"]
        cases.append(dict(name=name, key=key, attrs=attrs, bmad_line=src_line, output_line=g["line"],
                          tol=g["tol"], expected_vec=g["values"][:6]))
    json.dump(dict(source="regression_tests/tracking_method_test", e_tot=TM_E_TOT, charge=TM_CHARGE, start=TM_START,
                   cases=cases), open(os.path.join(HERE, "tracking_method_bmad_standard.json"), "w"), indent=1)

    m6 = parse_output_correct(os.path.join(REF, "regression_tests/mat6_calc_method_test/output.correct"))
    mcases = []
    for name, (key, attrs, src_line) in M6_ELEMENTS.items():
        rows = [m6["%s:Tracking:MatrixRow%d" % (name, i)] for i in range(1, 7)]
        vec0 = m6[name + ":Tracking:Vector"]
        mcases.append(dict(name=name, key=key, attrs=attrs, bmad_line=src_line, output_line=vec0["line"],
                           tol_matrix=max(r["tol"] for r in rows), tol_rows=[r["tol"] for r in rows], tol_vec0=vec0["tol"],
                           expected_mat6=[r["values"] for r in rows], expected_vec0=vec0["values"]))
    json.dump(dict(source="regression_tests/mat6_calc_method_test", e_tot=1e6, charge=1.0, start=TM_START, d_orb=1e-5,
                   cases=mcases), open(os.path.join(HERE, "mat6_calc_method_tracking.json"), "w"), indent=1)

    ap = parse_output_correct(os.path.join(REF, "regression_tests/aperture_test/output.correct"))
    grids = aperture_grids()
    acases = []
    for name, (key, attrs, src_line) in AP_ELEMENTS.items():
        for g, vecs in grids.items():
            st, un = ap["%s_S_%s" % (name, g)], ap["%s_U_%s" % (name, g)]
            acases.append(dict(name="%s_%s" % (name, g), key=key, attrs=attrs, bmad_line=src_line,
                               output_line=st["line"], vecs=vecs, expected_state=[int(v) for v in st["values"]],
                               expected_unstable=un["values"], tol=un["tol"]))
    json.dump(dict(source="regression_tests/aperture_test", particle_at="second_track_edge", cases=acases),
              open(os.path.join(HERE, "aperture_test_collimators.json"), "w"), indent=1)

    ct = parse_output_correct(os.path.join(REF, "regression_tests/coord_test/output.correct"))
    ccases = []
    for name, (key, attrs, src_line) in CT_ELEMENTS.items():
        st = ct["%s:O:1:D:1:Drift-Start-orb" % name]
        ccases.append(dict(name=name, key=key, attrs=attrs, bmad_line=src_line, output_line=st["line"],
                           tol=st["tol"], start=st["values"][:6],
                           expected={stage: ct["%s:O:1:D:1:Drift-%s-orb" % (name, stage)]["values"][:6]
                                     for stage in ("In:", "Xfer", "Out")}))
    json.dump(dict(source="regression_tests/coord_test", e_tot=1e8, charge=-1.0, cases=ccases),
              open(os.path.join(HERE, "coord_test_bend_offsets.json"), "w"), indent=1)

    fr = parse_output_correct(os.path.join(REF, "regression_tests/fringe_test/output.correct"))
    fcases = []
    for edge, tag in (("first_track_edge", "Up"), ("second_track_edge", "Dn")):
        rows = [fr["%s-Mat%d" % (tag, i)]["values"] for i in range(1, 7)]
        fcases.append(dict(edge=edge, tol=fr[tag + "-Orb"]["tol"], expected_dorb=fr[tag + "-Orb"]["values"],
                           expected_dmat=rows))
    json.dump(dict(source="regression_tests/fringe_test", e_tot=1e6, charge=-1.0, start=FR_START, element=FR_ELEMENT,
                   cases=fcases), open(os.path.join(HERE, "fringe_test_hwang.json"), "w"), indent=1)
    print("wrote", len(cases), "tracking_method cases and", len(fcases), "fringe cases")


if __name__ == "__main__":
    sys.exit(main())
