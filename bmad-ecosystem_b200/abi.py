"""ctypes mirror of include/bmadgpu.h (the C-ABI of the tracker).

The structures keep the field order and types of the C header; ``check_layout`` compares their
sizes with the values the compiled library reports, so a drift between the two fails loudly.
Enum values are Bmad's own (bmad/modules/bmad_struct.f90), so Fortran callers pass ele%key,
coord%state, ... unchanged.
"""
import ctypes as C
import math

N_POLE = 22          # 0:n_pole_maxx, n_pole_maxx = 21 (bmad_struct.f90:48)
N_MOMENTS = 28

# status codes
OK, EINVAL, ENOMEM, ECUDA, ETIMEDOUT, EUNSUPPORTED, EBUSY, ENOTFOUND = 0, -1, -2, -3, -4, -5, -6, -7
STATUS_NAMES = {0: "OK", -1: "EINVAL", -2: "ENOMEM", -3: "ECUDA", -4: "ETIMEDOUT",
                -5: "EUNSUPPORTED", -6: "EBUSY", -7: "ENOTFOUND"}

# element keys (bmad_struct.f90:1696-1710)
DRIFT, SBEND, QUADRUPOLE, SEXTUPOLE, RFCAVITY, MARKER = 1, 2, 3, 5, 9, 14
OCTUPOLE, MULTIPOLE, AB_MULTIPOLE, MONITOR, INSTRUMENT, PIPE, THICK_MULTIPOLE = 17, 19, 22, 31, 32, 44, 67
RCOLLIMATOR, ECOLLIMATOR = 35, 36
KICKER, HKICKER, VKICKER, ELSEPARATOR = 15, 33, 34, 10
# particle states (bmad_struct.f90:525-532)
ALIVE, LOST, LOST_NEG_X, LOST_POS_X, LOST_NEG_Y, LOST_POS_Y, LOST_Z, LOST_PZ = 1, 2, 3, 4, 5, 6, 7, 8
# locations (bmad_struct.f90:376-377)
UPSTREAM_END, DOWNSTREAM_END, INSIDE = 1, 2, 3
# ends (bmad_struct.f90:373-374)
ENTRANCE_END, EXIT_END, BOTH_ENDS, NO_END, CONTINUOUS = 1, 2, 3, 4, 5
# fringe types (bmad_struct.f90:27, 168-169)
FRINGE_NONE, FRINGE_SOFT_EDGE_ONLY, FRINGE_HARD_EDGE_ONLY, FRINGE_FULL = 1, 2, 3, 4
FRINGE_SAD_FULL, FRINGE_LINEAR_EDGE, FRINGE_BASIC_BEND = 5, 6, 7
# aperture types (bmad_struct.f90:158)
APERTURE_AUTO, APERTURE_RECTANGULAR, APERTURE_ELLIPTICAL = 1, 2, 3

# physical constants (sim_utils/interfaces/physical_constants.f90:12, 18, 34)
PI = 3.141592653589793238462643383279
C_LIGHT = 2.99792458e8
M_ELECTRON = 0.51099895069e6

_DOUBLE_FIELDS = (
    "l k1 k2 k3 g dg e1 e2 fint fintx hgap hgapx "
    "tilt ref_tilt roll x_offset y_offset z_offset x_pitch y_pitch "
    "hkick vkick x1_limit x2_limit y1_limit y2_limit "
    "voltage rf_frequency phi0 phi0_multipass ds_step r0_mag r0_elec delta_ref_time"
).split()


class Element(C.Structure):
    """bmadgpu_element: one tracked element; field names are Bmad's ele%value(...) names."""
    _fields_ = (
        [(n, C.c_int32) for n in ("key is_on fringe_type fringe_at aperture_at aperture_type "
                                  "num_steps scale_multipoles field_master exact_multipoles "
                                  "orientation reserved").split()]
        + [(n, C.c_double) for n in _DOUBLE_FIELDS]
        + [("a_pole", C.c_double * N_POLE), ("b_pole", C.c_double * N_POLE),
           ("a_pole_elec", C.c_double * N_POLE), ("b_pole_elec", C.c_double * N_POLE),
           ("fq1", C.c_double), ("fq2", C.c_double),
           ("px_aperture_width2", C.c_double), ("px_aperture_center", C.c_double),
           ("py_aperture_width2", C.c_double), ("py_aperture_center", C.c_double),
           ("z_aperture_width2", C.c_double), ("z_aperture_center", C.c_double),
           ("pz_aperture_width2", C.c_double), ("pz_aperture_center", C.c_double), ("kick", C.c_double)]
    )


class Param(C.Structure):
    """bmadgpu_param: lat_param_struct plus the bmad_com switches the path reads."""
    _fields_ = [("p0c", C.c_double), ("e_tot", C.c_double), ("mass", C.c_double),
                ("charge", C.c_double), ("max_aperture_limit", C.c_double),
                ("default_ds_step", C.c_double), ("aperture_limit_on", C.c_int32),
                ("absolute_time_tracking", C.c_int32), ("radiation_on", C.c_int32),
                ("reserved", C.c_int32)]


class Bunch(C.Structure):
    """bmadgpu_bunch: structure-of-arrays particle view (host or device pointers)."""
    _fields_ = [("n", C.c_int64), ("vec", C.c_void_p), ("beta", C.c_void_p), ("t", C.c_void_p),
                ("state", C.c_void_p), ("ix_ele", C.c_void_p), ("ix_turn", C.c_void_p),
                ("location", C.c_void_p)]


def default_element(key, **kw):
    """An Element with Bmad's defaults for `key` (set_ele_defaults.f90:36-37, 295-320;
    bmad_struct.f90:1509-1524), then the given attributes. fintx/hgapx follow fint/hgap unless
    given (bmad_parser_mod.f90:5238-5239)."""
    e = Element()
    e.key = key
    e.is_on = 1
    e.fringe_type = FRINGE_BASIC_BEND if key == SBEND else FRINGE_NONE
    e.fringe_at = BOTH_ENDS
    e.aperture_at = EXIT_END
    e.aperture_type = APERTURE_ELLIPTICAL if key == ECOLLIMATOR else APERTURE_RECTANGULAR
    e.scale_multipoles = 1
    e.exact_multipoles = 1   # off$
    e.orientation = 1
    poles = {}
    for k, v in kw.items():
        if k in ("a_pole", "b_pole", "a_pole_elec", "b_pole_elec"):
            poles[k] = v
        else:
            setattr(e, k, v)
    if key == SBEND:
        if "fintx" not in kw:
            e.fintx = e.fint
        if "hgapx" not in kw:
            e.hgapx = e.hgap
    for k, v in poles.items():
        arr = getattr(e, k)
        if isinstance(v, dict):
            for i, x in v.items():
                arr[int(i)] = x
        else:
            for i, x in enumerate(v):
                arr[i] = x
    return e


def electron_param(e_tot, **kw):
    """Param for an electron ring at total energy e_tot [eV]; p0c as convert_total_energy_to
    (bmad/code/convert_total_energy_to.f90) computes it."""
    p = Param()
    p.e_tot = float(e_tot)
    p.mass = M_ELECTRON
    p.p0c = math.sqrt(p.e_tot * p.e_tot - p.mass * p.mass)
    p.charge = -1.0
    p.max_aperture_limit = 1e3
    p.default_ds_step = 0.2
    p.aperture_limit_on = 1
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def element_array(elements):
    arr = (Element * len(elements))()
    for i, e in enumerate(elements):
        arr[i] = e
    return arr
