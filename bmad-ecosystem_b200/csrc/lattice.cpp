// lattice.cpp -- host-side element-table packer.
//
// Turns bmadgpu_element records (Bmad ele%value attributes) into the packed device table of
// table.h. This is the work Bmad's lattice bookkeeping does before tracking:
//   - tilt_tot / has_misalign:          bmad/code/attribute_bookkeeper.f90:146-170
//   - ds_step / num_steps (check_bend):  bmad/code/attribute_bookkeeper.f90:292-400,
//                                        forest/code/So_fitting.f90:3516-3548
//   - element a/b multipoles, b1 pull:   bmad/code/multipole_ele_to_ab.f90:31-678
//   - multipole kt <-> ab:               bmad/low_level/multipole1_{kt_to_ab,ab_to_kt}.f90
// and the per-element invariants the maps would otherwise recompute for every particle:
// bend-angle trig (track_a_bend.f90:134-160), Hwang edge coefficients (fringe_mod.f90:275-290),
// scaled kick coefficients (multipole_mod.f90:336-360), tilt cos/sin (tilt_coords.f90:40-41).

#include "lattice.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#if defined(BG_CR_MATH)
#include "crmath.cuh"
#endif

namespace bmadgpu {
namespace {

// The libm of the element invariants: correctly rounded in the product library (whose device
// maps are correctly rounded) and in the test-only host builds made with BG_CR_MATH; the host's
// libm in the other test-only host builds, which the oracle's default mode matches.
#if defined(BG_CR_MATH)
double l_sin(double x) { return cr::sin(x); }
double l_cos(double x) { return cr::cos(x); }
double l_atan2(double y, double x) { return cr::atan2(y, x); }
#else
double l_sin(double x) { return std::sin(x); }
double l_cos(double x) { return std::cos(x); }
double l_atan2(double y, double x) { return std::atan2(y, x); }
#endif

const double kPi = 3.141592653589793238462643383279;
const int kNPole = BMADGPU_N_POLE;

int nint(double x) { return (int)std::lround(x); }

int max_nonzero(const double* a, const double* b, int ub) {
  for (int i = ub; i >= 0; i--)
    if (a[i] != 0 || (b && b[i] != 0)) return i;
  return -1;
}

bool any_nonzero(const double* a, int n) {
  for (int i = 0; i < n; i++)
    if (a[i] != 0) return true;
  return false;
}

double factorial(int n) {
  double f = 1;
  for (int i = 2; i <= n; i++) f *= i;
  return f;
}

double sinc0(double x) { return std::fabs(x) < 1e-8 ? 1.0 : l_sin(x) / x; }
double cosc0(double x) {
  if (std::fabs(x) < 1e-8) return 0.5;
  double s = sinc0(x / 2);
  return 0.5 * (s * s);
}
double sincc0(double x) {
  double x2 = x * x;
  if (std::fabs(x) < 0.1)
    return 1.0 / 6.0 + x2 * (-1.0 / 120.0 + x2 * (1.0 / 5040.0 + x2 * (-1.0 / 362880.0)));
  return (x - l_sin(x)) / (x * x2);
}

struct Fail {
  int code;
  std::string msg;
};

bool key_supported(int key) {
  switch (key) {
    case BMADGPU_DRIFT: case BMADGPU_SBEND: case BMADGPU_QUADRUPOLE: case BMADGPU_SEXTUPOLE:
    case BMADGPU_RFCAVITY: case BMADGPU_MARKER: case BMADGPU_OCTUPOLE: case BMADGPU_MULTIPOLE:
    case BMADGPU_AB_MULTIPOLE: case BMADGPU_MONITOR: case BMADGPU_INSTRUMENT: case BMADGPU_PIPE:
    case BMADGPU_THICK_MULTIPOLE: case BMADGPU_RCOLLIMATOR: case BMADGPU_ECOLLIMATOR:
    case BMADGPU_KICKER: case BMADGPU_HKICKER: case BMADGPU_VKICKER: case BMADGPU_ELSEPARATOR:
      return true;
  }
  return false;
}

// has_hkick_attributes (attribute_mod.f90:746-765, 1879) for the keys on the path
bool key_has_hkick(int key) {
  switch (key) {
    case BMADGPU_QUADRUPOLE: case BMADGPU_SBEND: case BMADGPU_SEXTUPOLE: case BMADGPU_OCTUPOLE:
    case BMADGPU_THICK_MULTIPOLE: case BMADGPU_RFCAVITY: case BMADGPU_MONITOR: case BMADGPU_INSTRUMENT:
    case BMADGPU_RCOLLIMATOR: case BMADGPU_ECOLLIMATOR: case BMADGPU_KICKER:
      return true;
  }
  return false;
}

// Element magnetic a/b multipoles in the body frame with the non-multipole kick terms included
// (multipole_ele_to_ab with use_ele_tilt = F, include_kicks = include_kicks$).
void mag_ab(const bmadgpu_element& e, double tilt_tot, double ref_tilt_tot, double* a, double* b,
            int* ix_pole_max) {
  for (int i = 0; i < kNPole; i++) { a[i] = 0; b[i] = 0; }
  *ix_pole_max = -1;
  if (!e.is_on || e.key == BMADGPU_PIPE) return;
  if (e.key == BMADGPU_MULTIPOLE) {
    for (int n = 0; n < kNPole; n++) {
      double knl = e.a_pole[n], tn = e.b_pole[n];
      if (knl == 0) continue;
      double angle = -tn * (n + 1);
      b[n] = (knl * l_cos(angle) - 0.0 * l_sin(angle)) / factorial(n);
      a[n] = (knl * l_sin(angle) + 0.0 * l_cos(angle)) / factorial(n);
    }
    *ix_pole_max = max_nonzero(a, b, kNPole - 1);
    return;
  }
  // convert_this_ab (multipole_ele_to_ab.f90:472-600), scale_multipoles with r0_mag
  if (any_nonzero(e.a_pole, kNPole) || any_nonzero(e.b_pole, kNPole)) {
    for (int i = 0; i < kNPole; i++) { a[i] = e.a_pole[i]; b[i] = e.b_pole[i]; }
    if (e.scale_multipoles) {
      double cnst = 1;
      int ref_exp = 0;
      bool scale = true;
      switch (e.key) {
        case BMADGPU_SBEND: cnst = e.l * (e.g + e.dg); ref_exp = 0; break;
        case BMADGPU_QUADRUPOLE: cnst = e.k1 * e.l; ref_exp = 1; break;
        case BMADGPU_SEXTUPOLE: cnst = e.k2 * e.l; ref_exp = 2; break;
        case BMADGPU_OCTUPOLE: cnst = e.k3 * e.l; ref_exp = 3; break;
        case BMADGPU_KICKER: case BMADGPU_ELSEPARATOR:
          if (e.hkick == 0) cnst = e.vkick;
          else if (e.vkick == 0) cnst = e.hkick;
          else cnst = std::sqrt(e.hkick * e.hkick + e.vkick * e.vkick);
          ref_exp = 0;
          break;
        case BMADGPU_HKICKER: case BMADGPU_VKICKER: cnst = e.kick; ref_exp = 0; break;
        default: scale = false;
      }
      if (scale) {
        if (e.r0_mag == 0) {
          for (int i = 0; i < kNPole; i++) { a[i] = cnst * a[i]; b[i] = cnst * b[i]; }
        } else {
          double factor = cnst * std::pow(e.r0_mag, ref_exp + 1);
          for (int i = 0; i < kNPole; i++) {
            factor = factor / e.r0_mag;
            a[i] = factor * a[i];
            b[i] = factor * b[i];
          }
        }
      }
    }
  }
  // this_ele_non_multipoles (multipole_ele_to_ab.f90:326-405)
  double ak[4] = {0, 0, 0, 0}, bk[4] = {0, 0, 0, 0};
  if (e.key == BMADGPU_HKICKER) {         // multipole_ele_to_ab.f90:339-346
    bk[0] = -e.kick;
  } else if (e.key == BMADGPU_VKICKER) {
    ak[0] = e.kick;
  } else if (e.key == BMADGPU_KICKER) {
    bk[0] = -e.hkick;
    ak[0] = e.vkick;
  } else if (e.key == BMADGPU_ELSEPARATOR) {
    // the separator's kick is its electric field (track_this_elsep), not a multipole
  } else if (key_has_hkick(e.key) && (e.hkick != 0 || e.vkick != 0)) {
    double tilt = (e.key == BMADGPU_SBEND) ? ref_tilt_tot : tilt_tot;
    if (tilt != 0) {
      double c = l_cos(tilt), s = l_sin(tilt);
      bk[0] = -e.hkick * c - e.vkick * s;
      ak[0] = -e.hkick * s + e.vkick * c;
    } else {
      bk[0] = -e.hkick;
      ak[0] = e.vkick;
    }
  }
  switch (e.key) {
    case BMADGPU_QUADRUPOLE: bk[1] = e.k1 * e.l; break;
    case BMADGPU_SBEND:
      bk[0] = bk[0] + e.dg * e.l;
      bk[1] = e.k1 * e.l;
      bk[2] = e.k2 * e.l / 2.0;
      break;
    case BMADGPU_SEXTUPOLE: bk[2] = e.k2 * e.l / 2.0; break;
    case BMADGPU_OCTUPOLE: bk[3] = e.k3 * e.l / 6.0; break;
  }
  for (int i = 0; i < 4; i++) { a[i] = a[i] + ak[i]; b[i] = b[i] + bk[i]; }
  *ix_pole_max = max_nonzero(a, b, kNPole - 1);
}

// tilt_this_multipole(+1) for ab_multipole elements (use_ele_tilt = T)
void tilt_ab(double tilt, double* a, double* b, int ix_pole_max) {
  if (tilt == 0) return;
  for (int n = 0; n <= ix_pole_max; n++) {
    if (a[n] == 0 && b[n] == 0) continue;
    double an = a[n], bn = b[n];
    double c = l_cos((n + 1) * tilt), s = l_sin((n + 1) * tilt);
    b[n] = bn * c + an * s;
    a[n] = -bn * s + an * c;
  }
}

// multipole1_ab_to_kt, bmad/low_level/multipole1_ab_to_kt.f90:17
void ab_to_kt(double an, double bn, int n, double* knl, double* tn) {
  if (an == 0 && bn == 0) { *knl = 0; *tn = 0; return; }
  *knl = factorial(n) * std::sqrt(an * an + bn * bn);
  *tn = -l_atan2(an, bn) / (n + 1);
  if (2 * (n + 1) * std::fabs(*tn) > kPi) {
    *knl = -*knl;
    double sgn = (*tn < 0) ? -1.0 : 1.0;
    *tn = sgn * (std::fabs(*tn) - kPi / (n + 1));
  }
}

// pull_this_b1 (multipole_ele_to_ab.f90:664-676)
double pull_b1(double* a, double* b, int* ix_pole_max) {
  double b1 = b[1];
  b[1] = 0;
  if (*ix_pole_max > 1) return b1;
  *ix_pole_max = max_nonzero(a, b, 1);
  return b1;
}

// check_bend (forest/code/So_fitting.f90:3516-3548): integration steps for a given error budget.
void check_bend(double xl, double ggi, double rhoi, double xbend1, double gf[8], int* met) {
  double gg = (double)(long long)ggi;
  if (gg == 0.0) gg = 1.0;
  const double co[8] = {0, 0, 1.0 / 12.0, 0, 0.17, 0, 0.17e-1, 0};
  for (int i = 0; i < 8; i++) gf[i] = 0;
  for (int i = 3; i <= 7; i += 2) {
    double ar = i - 1;
    gf[i] = std::pow(co[i - 1] / xbend1, 1.0 / ar) * std::fabs(rhoi) * xl;
    if (gf[i] < gg) gf[i] = gg;
  }
  gf[2] = gf[3];
  gf[4] = gf[5] * 3;
  gf[6] = gf[7] * 7;
  *met = 2;
  if (gf[4] < gf[2]) *met = 4;
  if (gf[6] < gf[4] && gf[6] < gf[2]) *met = 6;
}

// ds_step and num_steps as attribute_bookkeeper.f90:292-400 resolves them.
void resolve_steps(const bmadgpu_element& e, const bmadgpu_param& p, double tilt_tot, double* ds_out,
                   int* n_out) {
  double ds_step = e.ds_step;
  double num_steps = e.num_steps;
  if (num_steps == 0 && e.key == BMADGPU_RFCAVITY) num_steps = 10;  // set_ele_defaults.f90:319
  double L = e.l;
  if (ds_step == 0 && num_steps == 0) {
    switch (e.key) {
      case BMADGPU_DRIFT: case BMADGPU_PIPE: case BMADGPU_INSTRUMENT: case BMADGPU_MONITOR:
      case BMADGPU_RCOLLIMATOR: case BMADGPU_ECOLLIMATOR:
        num_steps = 1;
        ds_step = L;
        break;
      case BMADGPU_SBEND: case BMADGPU_QUADRUPOLE: case BMADGPU_SEXTUPOLE:
        if (L != 0) {
          double a[kNPole], b[kNPole], knl[kNPole];
          int ix;
          mag_ab(e, tilt_tot, e.ref_tilt, a, b, &ix);
          for (int n = 0; n < kNPole; n++)
            knl[n] = (a[n] == 0 && b[n] == 0) ? 0.0 : factorial(n) * std::sqrt(a[n] * a[n] + b[n] * b[n]);
          double bend_factor = knl[0] / L;
          double radius0 = e.r0_mag == 0 ? 0.01 : e.r0_mag;
          double quad_factor;
          if (e.key == BMADGPU_SBEND) {
            bend_factor = bend_factor + std::max(std::fabs(e.g), std::fabs(e.g + e.dg));
            quad_factor = knl[1] + knl[2] * radius0 + L * (bend_factor * bend_factor);
          } else if (e.key == BMADGPU_QUADRUPOLE) {
            quad_factor = 50 * (knl[1] + L * (bend_factor * bend_factor));
          } else {
            quad_factor = knl[2] * radius0 + L * (bend_factor * bend_factor);
          }
          double gf[8];
          int met;
          check_bend(L, quad_factor, bend_factor, 1e-8, gf, &met);
          int ixm = std::min(met, 4);
          num_steps = std::max(nint(gf[ixm + 1]), 1);
          ds_step = std::fabs(L) / num_steps;
        }
        break;
      default:
        break;
    }
  }
  if (ds_step <= 0) {
    if (num_steps <= 0 || std::fabs(L) == 0) ds_step = p.default_ds_step;
    else ds_step = std::fabs(L) / num_steps;
  }
  *ds_out = ds_step;
  *n_out = std::max(1, nint(std::fabs(L / ds_step)));
}

// ---- electric multipoles and the misaligned-bend frame ----------------------------------------

// at_this_ele_end, bmad/code/at_this_ele_end.f90:16-61 (now_at: entrance or exit end)
bool at_ele_end(int now_at, int where_at) {
  if (where_at == BMADGPU_NO_END) return false;
  if (where_at == BMADGPU_CONTINUOUS || where_at == 7) return true;
  if (now_at == BMADGPU_ENTRANCE_END) return where_at == BMADGPU_ENTRANCE_END || where_at == BMADGPU_BOTH_ENDS;
  return where_at == BMADGPU_EXIT_END || where_at == BMADGPU_BOTH_ENDS;
}

// Electric a/b multipoles (multipole_ele_to_ab with pole_type = electric: convert_this_ab with
// r0_elec scaling, multipole_ele_to_ab.f90:472-520); returns ix_elec_max.
int elec_ab(const bmadgpu_element& e, double* a, double* b) {
  for (int i = 0; i < kNPole; i++) { a[i] = 0; b[i] = 0; }
  if (!e.is_on || e.key == BMADGPU_PIPE || e.key == BMADGPU_MULTIPOLE) return -1;
  for (int i = 0; i < kNPole; i++) { a[i] = e.a_pole_elec[i]; b[i] = e.b_pole_elec[i]; }
  if (max_nonzero(a, b, kNPole - 1) < 0) return -1;
  if (e.scale_multipoles) {
    const double radius = e.r0_elec;
    if (radius != 0 && radius != 1) {
      double factor = radius;
      for (int n = 0; n < kNPole; n++) {
        factor = factor / radius;
        a[n] = factor * a[n];
        b[n] = factor * b[n];
      }
    }
  }
  return max_nonzero(a, b, kNPole - 1);
}

// The extra block (table.h) of a quadrupole, sextupole, octupole, thick multipole or sbend, or an
// empty vector when the element needs none. Straight elements: apply_element_edge_kick runs when
// init_fringe_info finds a fringe (fringe_type != none with fringe_at != no_end, or electric
// multipoles; init_fringe_info.f90:22-55); bends: always, with the block only for electric
// multipoles or fringe_type full (the Hwang edges are in the bend's own block). At each end the
// edge acts when at_this_ele_end(fringe_at); fringe_here adds fringe_type != none
// (fringe_here.f90:15-35); the electric fringe needs a length (apply_element_edge_kick.f90:290);
// hard_multipole_edge_kick acts for full and hard_edge_only (not on bends), soft_quadrupole_
// edge_kick for full and soft_edge_only (fringe_mod.f90:556-577, 692-722), exact_bend_edge_kick
// for full (:40-99). s_half / s_full: the electric kick scales of the element's loop.
std::vector<double> extra_block(const bmadgpu_element& e, const bmadgpu_param& p, const double* a, const double* b,
                                int ix_elec_max, double s_half, double s_full) {
  const bool raw_elec = any_nonzero(e.a_pole_elec, kNPole) || any_nonzero(e.b_pole_elec, kNPole);
  const int ft = e.fringe_type;
  const bool bend = e.key == BMADGPU_SBEND;
  if (bend) {
    if (ix_elec_max < 0 && ft != BMADGPU_FRINGE_FULL) return {};
  } else {
    // init_fringe_info: an elseparator always has a fringe (its longitudinal field)
    const bool has_fringe = (ft != BMADGPU_FRINGE_NONE && e.fringe_at != BMADGPU_NO_END) || raw_elec ||
                            e.key == BMADGPU_ELSEPARATOR;
    if (!has_fringe) return {};
  }
  auto bits = [&](int end) {
    if (!at_ele_end(end, e.fringe_at)) return 0.0;
    int m = EX_CALL;
    if (ix_elec_max > -1 && e.l != 0) m |= EX_ELEC;
    if (ft != BMADGPU_FRINGE_NONE) {
      const bool hard = ft == BMADGPU_FRINGE_FULL || (ft == BMADGPU_FRINGE_HARD_EDGE_ONLY && !bend);
      if (hard && (bend || e.key == BMADGPU_QUADRUPOLE || e.key == BMADGPU_SEXTUPOLE)) m |= EX_HARD;
      if ((ft == BMADGPU_FRINGE_FULL || ft == BMADGPU_FRINGE_SOFT_EDGE_ONLY) && e.key == BMADGPU_QUADRUPOLE)
        m |= EX_SOFT;
      if (bend && ft == BMADGPU_FRINGE_FULL) m |= EX_EXACT;
    }
    if (e.key == BMADGPU_ELSEPARATOR && e.l != 0) m |= EX_ESEP;
    return (double)m;
  };
  const int n_elec = ix_elec_max + 1;
  std::vector<double> blk = {(double)n_elec, s_half, s_full, bits(BMADGPU_ENTRANCE_END), bits(BMADGPU_EXIT_END),
                             1.0 * p.charge, -1.0 * p.charge, p.mass / p.p0c,
                             e.key == BMADGPU_SEXTUPOLE ? 2.0 : 1.0, e.key == BMADGPU_SEXTUPOLE ? e.k2 : e.k1,
                             e.k1, e.fq1, e.fq2,
                             e.is_on ? e.g + e.dg : 0.0, p.p0c / p.e_tot,
                             1 * e.e1, 1 * e.fint, e.hgap, 1 * e.e2, 1 * e.fintx, e.hgapx,
                             0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0,   // elseparator steps, set by the caller
                             e.l != 0 ? 1.0 * p.charge * (p.p0c / e.l) : 0.0,
                             e.l != 0 ? -1.0 * p.charge * (p.p0c / e.l) : 0.0, e.hkick, e.vkick};
  for (int n = 0; n < n_elec; n++) blk.insert(blk.end(), {b[n], a[n]});
  return blk;
}

typedef double Mat3[3][3];

// Fortran matmul of 3x3 matrices, j-order summation
void matmul3(const Mat3 a, const Mat3 b, Mat3 out) {
  Mat3 t;
  for (int i = 0; i < 3; i++)
    for (int k = 0; k < 3; k++) {
      double acc = 0;
      for (int j = 0; j < 3; j++) acc = acc + a[i][j] * b[j][k];
      t[i][k] = acc;
    }
  std::memcpy(out, t, sizeof(t));
}

// floor_angles_to_w_mat (bmad/geometry/floor_angles_to_w_mat.f90), or its inverse
void w_mat_angles(double theta, double phi, bool inverse, Mat3 w, double psi = 0.0) {
  const double s_the = l_sin(theta), c_the = l_cos(theta);
  const double s_phi = l_sin(phi), c_phi = l_cos(phi);
  const double s_psi = l_sin(psi), c_psi = l_cos(psi);
  const double m[9] = {c_the * c_psi - s_the * s_phi * s_psi, -c_the * s_psi - s_the * s_phi * c_psi,
                       s_the * c_phi, c_phi * s_psi, c_phi * c_psi, s_phi,
                       -s_the * c_psi - c_the * s_phi * s_psi, s_the * s_psi - c_the * s_phi * c_psi,
                       c_the * c_phi};
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) w[i][j] = inverse ? m[3 * j + i] : m[3 * i + j];
}

// cos_one (sim_utils/special_functions/cos_one.f90:16-27)
double cos_one(double angle) {
  const double s = l_sin(angle / 2);
  return -2 * (s * s);
}

// rotate_vec / rotate_mat about the x (1), y (2) or z (3) axis, sim_utils/math/rotation_3d_mod.f90:
// 737-845 (the matrix rotated from the left)
void rotate_vec(double v[3], int axis, double angle) {
  if (angle == 0) return;
  const double ca = l_cos(angle), sa = l_sin(angle);
  if (axis == 1) {
    const double a = ca * v[1] - sa * v[2], b = sa * v[1] + ca * v[2];
    v[1] = a;
    v[2] = b;
  } else if (axis == 2) {
    const double a = sa * v[2] + ca * v[0], b = ca * v[2] - sa * v[0];
    v[0] = a;
    v[2] = b;
  } else {
    const double a = ca * v[0] - sa * v[1], b = sa * v[0] + ca * v[1];
    v[0] = a;
    v[1] = b;
  }
}
void rotate_mat(Mat3 m, int axis, double angle) {
  if (angle == 0) return;
  const double ca = l_cos(angle), sa = l_sin(angle);
  for (int k = 0; k < 3; k++) {
    if (axis == 1) {
      const double a = ca * m[1][k] - sa * m[2][k], b = sa * m[1][k] + ca * m[2][k];
      m[1][k] = a;
      m[2][k] = b;
    } else if (axis == 2) {
      const double a = sa * m[2][k] + ca * m[0][k], b = ca * m[2][k] - sa * m[0][k];
      m[0][k] = a;
      m[2][k] = b;
    } else {
      const double a = ca * m[0][k] - sa * m[1][k], b = sa * m[0][k] + ca * m[1][k];
      m[0][k] = a;
      m[1][k] = b;
    }
  }
}

// One end of the bend frame: the rotation chain w of the floor position and the steps acting on
// its position r, recorded in the reference's order (offset_particle.f90:204-257, 399-457).
struct FrameEnd {
  Mat3 w = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  std::vector<double> steps;
  int n = 0;
  void step(int op, const double* v1, const Mat3 m, const double* v2) {
    double st[BF_STEP] = {0};
    st[0] = op;
    for (int i = 0; i < 3; i++) {
      if (v1) st[1 + i] = v1[i];
      if (v2) st[13 + i] = v2[i];
    }
    if (m)
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) st[4 + 3 * i + j] = m[i][j];
    steps.insert(steps.end(), st, st + BF_STEP);
    n++;
  }
  void apply_w(const Mat3 m, int extra = 0, const double* v1 = nullptr) {  // r = m (r - v1), w = m w
    step(FS_MAT | extra, v1, m, nullptr);
    matmul3(m, w, w);
  }
  // bend_shift, bmad/geometry/bend_shift.f90:19-61 (has_tilt: the optional ref_tilt is present)
  void bend_shift(double g, double delta_s, bool has_tilt = false, double ref_tilt = 0) {
    const double angle = delta_s * g;
    if (angle == 0) {
      const double v[3] = {0, 0, delta_s};
      step(FS_SUBZ, v, nullptr, nullptr);
      return;
    }
    const double tlt = has_tilt ? ref_tilt : 0.0;
    Mat3 S = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    if (tlt != 0) {
      rotate_mat(S, 3, -ref_tilt);
      rotate_mat(S, 2, angle);
      rotate_mat(S, 3, ref_tilt);
    } else {
      rotate_mat(S, 2, angle);
    }
    double L[3] = {cos_one(angle) / g, 0.0 / g, -l_sin(angle) / g};
    if (has_tilt) rotate_vec(L, 3, ref_tilt);
    step(FS_MAT | FS_ADD, nullptr, S, L);
    matmul3(S, w, w);
  }
};

// The bend frame block of a bend with offsets, pitches, z_offset or roll. With g != 0, a ref_tilt
// or a roll, the bend_shift geometry, with the misalignment of ele_misalignment_L_S_calc
// (bmad/geometry/ele_misalignment_L_S_calc.f90:16-50: the offsets moved by the roll about the
// chord, the rotation floor_angles_to_w_mat(x_pitch, y_pitch, roll)); otherwise the straight
// transform of offset_particle (offset_particle.f90:239-245, 279-282, 437-443, 477-480), written
// as the same kind of steps.
std::vector<double> bend_frame_block(const bmadgpu_element& e) {
  const double length = e.l, L_half = 0.5 * length, g = e.g, rt = e.ref_tilt, roll = e.roll;
  double L_mis[3] = {e.x_offset, e.y_offset, e.z_offset};
  const double ds_set = L_half - 0.0, ds_unset = L_half - length;
  FrameEnd in, out;
  if (g != 0 || rt != 0 || roll != 0) {
    if (roll != 0) {  // angle = l g, rho = 1/g (0 for g = 0), attribute_bookkeeper.f90:763-770
      const double angle = e.l * g, rho = (g == 0) ? 0.0 : 1 / g;
      double Lc[3] = {rho * cos_one(angle / 2), rho * 0.0, rho * l_sin(angle / 2)};
      rotate_vec(Lc, 2, angle / 2);
      rotate_vec(Lc, 3, rt);
      for (int i = 0; i < 3; i++) L_mis[i] = L_mis[i] - Lc[i];
      rotate_vec(Lc, 3, roll);
      for (int i = 0; i < 3; i++) L_mis[i] = L_mis[i] + Lc[i];
    }
    in.bend_shift(g, 1 * ds_set, true, rt);
    Mat3 ws, wt;
    w_mat_angles(e.x_pitch, e.y_pitch, false, ws, roll);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) wt[i][j] = ws[j][i];
    in.apply_w(wt, FS_SUB, L_mis);
    if (rt != 0) {
      in.bend_shift(g, -L_half, true, rt);
      const double c = l_cos(-rt), s = l_sin(-rt);   // w_mat_for_tilt (w_mat_for_tilt.f90:14-38)
      const Mat3 wm = {{c, -s, 0.0}, {s, c, 0.0}, {0.0, 0.0, 1.0}};
      in.apply_w(wm);
      in.bend_shift(g, L_half);
    }
    in.bend_shift(g, -1 * 1 * L_half);
    const double zs[3] = {0, 0, (1 - 1 * 1) * L_half};
    in.step(FS_ADDZ, nullptr, nullptr, zs);

    out.bend_shift(g, ds_unset);
    if (rt != 0) {
      out.bend_shift(g, -L_half);
      const double c = l_cos(rt), s = l_sin(rt);
      const Mat3 wm = {{c, -s, 0.0}, {s, c, 0.0}, {0.0, 0.0, 1.0}};
      out.apply_w(wm);
      out.bend_shift(g, L_half, true, rt);
    }
    out.apply_w(ws);
    out.step(FS_ADD, nullptr, nullptr, L_mis);
    out.bend_shift(g, 1 * 1 * L_half, true, rt);
    const double zu[3] = {0, 0, (1 + 1 * 1) * L_half};
    out.step(FS_ADDZ, nullptr, nullptr, zu);
  } else {
    Mat3 winv, ws;
    w_mat_angles(e.x_pitch, e.y_pitch, true, winv);
    w_mat_angles(e.x_pitch, e.y_pitch, false, ws);
    const double v_in[3] = {e.x_offset, e.y_offset, e.z_offset + 1 * ds_set};
    in.step(FS_SUB | FS_MAT, v_in, winv, nullptr);
    std::memcpy(in.w, winv, sizeof(Mat3));
    const double zs[3] = {0, 0, L_half};
    in.step(FS_ADDZ, nullptr, nullptr, zs);
    const double v_out[3] = {0, 0, ds_unset};
    out.step(FS_SUBZ, v_out, nullptr, nullptr);
    const double add[3] = {e.x_offset, e.y_offset, e.z_offset + L_half};
    out.step(FS_MAT | FS_ADD, nullptr, ws, add);
    std::memcpy(out.w, ws, sizeof(Mat3));
  }
  std::vector<double> blk = {(double)in.n, (double)out.n, (1 - 1) * L_half, (1 + 1) * L_half};
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) blk.push_back(in.w[i][j]);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) blk.push_back(out.w[i][j]);
  blk.insert(blk.end(), in.steps.begin(), in.steps.end());
  blk.insert(blk.end(), out.steps.begin(), out.steps.end());
  return blk;
}

struct Packer {
  std::vector<EleHdr> hdr;
  std::vector<ApRec> ap;
  std::vector<double> pool;
  std::map<std::vector<double>, uint32_t> dedupe;
  std::map<std::vector<double>, uint16_t> ap_dedupe;

  uint32_t add_block(const std::vector<double>& blk) {
    if (blk.empty()) return 0;
    auto it = dedupe.find(blk);
    if (it != dedupe.end()) return it->second;
    // keep blocks 16-byte aligned so a block can be fetched with 16-byte loads
    if (pool.size() % 2) pool.push_back(0.0);
    uint32_t off = (uint32_t)pool.size();
    pool.insert(pool.end(), blk.begin(), blk.end());
    dedupe[blk] = off;
    return off;
  }
  uint16_t add_ap(const ApRec& r) {
    std::vector<double> k = {r.x1_lim, r.x2_lim, r.y1_lim, r.y2_lim, r.win_kind};
    k.insert(k.end(), r.win, r.win + 8);
    auto it = ap_dedupe.find(k);
    if (it != ap_dedupe.end()) return it->second;
    uint16_t ix = (uint16_t)ap.size();
    ap.push_back(r);
    ap_dedupe[k] = ix;
    return ix;
  }
};

void push_kicks(std::vector<double>& blk, const double* a, const double* b, int n_pole, double scale) {
  for (int n = 0; n < n_pole; n++) {
    blk.push_back(scale * b[n]);
    blk.push_back(scale * a[n]);
  }
}

// True if the two kick arrays starting at blk[off] (n_pole (b_n, a_n) pairs each, as the device
// reads them) hold only normal multipoles from order 2 up: every a_n zero and b_0 = b_1 = 0.
bool kicks_b_from2(const std::vector<double>& blk, size_t off, int n_pole) {
  if (n_pole < 3) return false;
  for (int arr = 0; arr < 2; arr++)
    for (int n = 0; n < n_pole; n++) {
      const double bn = blk[off + 2 * (arr * n_pole + n)], an = blk[off + 2 * (arr * n_pole + n) + 1];
      if (an != 0 || (n < 2 && bn != 0)) return false;
    }
  return true;
}

}  // namespace

void build_cmulti_tables(double cm[22][22], double cf[22][22]) {
  // c_multi.f90:38-63: binomials normalised by n!, sign - for m mod 4 in {0, 3}
  double c[22][22], nf[22];
  for (int i = 0; i < 22; i++)
    for (int j = 0; j < 22; j++) c[i][j] = 0;
  c[0][0] = 1;
  for (int in = 1; in < 22; in++) {
    c[in][0] = 1;
    c[in][in] = 1;
    for (int im = 1; im <= in - 1; im++) c[in][im] = c[in - 1][im - 1] + c[in - 1][im];
  }
  nf[0] = 1;
  for (int in = 0; in < 22; in++) {
    if (in > 0) nf[in] = in * nf[in - 1];
    for (int im = 0; im <= in; im++) {
      c[in][im] = c[in][im] / nf[in];
      if (im % 4 == 0) c[in][im] = -c[in][im];
      if (im % 4 == 3) c[in][im] = -c[in][im];
    }
  }
  for (int i = 0; i < 22; i++)
    for (int j = 0; j < 22; j++) {
      cf[i][j] = c[i][j];
      cm[i][j] = c[i][j] * nf[i];
    }
}

int pack_lattice(const bmadgpu_element* eles, int n_ele, const bmadgpu_param& p, PackedLattice& out,
                 std::string& err) {
  try {
    if (n_ele <= 0 || n_ele > 0xFFFFFF) throw Fail{BMADGPU_EINVAL, "n_ele out of range"};
    if (p.absolute_time_tracking) throw Fail{BMADGPU_EUNSUPPORTED, "absolute_time_tracking is not on the path"};
    if (p.radiation_on) throw Fail{BMADGPU_EUNSUPPORTED, "radiation/spin/wakes are not on the path"};
    if (!(p.p0c > 0) || !(p.e_tot > p.mass) || !(p.mass > 0))
      throw Fail{BMADGPU_EINVAL, "param: need p0c > 0, e_tot > mass > 0"};
    Packer pk;
    out.n_step.assign(n_ele, 1);
    out.ds_step.assign(n_ele, 0.0);
    double turn_ref = 0;
    for (int i = 0; i < n_ele; i++) {
      const bmadgpu_element& e = eles[i];
      auto fail = [&](int code, const std::string& m) {
        throw Fail{code, "element " + std::to_string(i) + " (key " + std::to_string(e.key) + "): " + m};
      };
      if (!key_supported(e.key)) fail(BMADGPU_EUNSUPPORTED, "element type not on the bmad_standard path");
      if (e.orientation != 1 && e.orientation != 0) fail(BMADGPU_EUNSUPPORTED, "orientation -1");
      if (e.field_master) fail(BMADGPU_EUNSUPPORTED, "field_master = T");
      if (e.exact_multipoles != 0 && e.exact_multipoles != 1) fail(BMADGPU_EUNSUPPORTED, "exact_multipoles");
      const bool raw_elec = any_nonzero(e.a_pole_elec, kNPole) || any_nonzero(e.b_pole_elec, kNPole);
      if (raw_elec && e.is_on && e.key != BMADGPU_MULTIPOLE && e.key != BMADGPU_QUADRUPOLE &&
          e.key != BMADGPU_SEXTUPOLE && e.key != BMADGPU_OCTUPOLE && e.key != BMADGPU_THICK_MULTIPOLE &&
          e.key != BMADGPU_SBEND)
        fail(BMADGPU_EUNSUPPORTED, "electric multipoles on this element type");
      if (e.key == BMADGPU_MULTIPOLE && any_nonzero(e.a_pole_elec, kNPole))
        fail(BMADGPU_EUNSUPPORTED, "multipole ksl");
      // convert_this_ab has no scale for other keys (multipole_ele_to_ab.f90:534-580)
      if (e.scale_multipoles && (any_nonzero(e.a_pole, kNPole) || any_nonzero(e.b_pole, kNPole)) &&
          (e.key == BMADGPU_MONITOR || e.key == BMADGPU_INSTRUMENT || e.key == BMADGPU_RCOLLIMATOR ||
           e.key == BMADGPU_ECOLLIMATOR || e.key == BMADGPU_DRIFT || e.key == BMADGPU_MARKER))
        fail(BMADGPU_EUNSUPPORTED, "scaled multipoles on an element type without a reference strength");
      if (e.x_pitch != 0 || e.y_pitch != 0 || e.z_offset != 0)
        if (e.key == BMADGPU_MULTIPOLE || e.key == BMADGPU_AB_MULTIPOLE)
          fail(BMADGPU_EUNSUPPORTED, "pitch / z_offset misalignment of a thin multipole");
      if (e.key == BMADGPU_SBEND && e.tilt != 0) fail(BMADGPU_EUNSUPPORTED, "sbend tilt (use ref_tilt)");

      if (e.key != BMADGPU_SBEND && e.ref_tilt != 0) fail(BMADGPU_EUNSUPPORTED, "ref_tilt on a non-bend");
      if (e.key == BMADGPU_RFCAVITY && (e.hkick != 0 || e.vkick != 0))
        fail(BMADGPU_EUNSUPPORTED, "rfcavity hkick/vkick");
      if (!key_has_hkick(e.key) && (e.hkick != 0 || e.vkick != 0) && e.key != BMADGPU_DRIFT &&
          e.key != BMADGPU_ELSEPARATOR)
        fail(BMADGPU_EUNSUPPORTED, "hkick/vkick on this element type");
      if (e.aperture_type != BMADGPU_APERTURE_RECTANGULAR && e.aperture_type != BMADGPU_APERTURE_AUTO &&
          e.aperture_type != BMADGPU_APERTURE_ELLIPTICAL)
        fail(BMADGPU_EUNSUPPORTED, "aperture_type");
      if (e.aperture_at < 1 || e.aperture_at > 4) fail(BMADGPU_EUNSUPPORTED, "aperture_at");

      double tilt_tot = (e.key == BMADGPU_SBEND) ? 0.0 : e.tilt;
      const bool pitched = e.x_pitch != 0 || e.y_pitch != 0 || e.z_offset != 0;
      const bool offset = e.x_offset != 0 || e.y_offset != 0 || pitched || (e.key == BMADGPU_SBEND && e.roll != 0);
      bool has_misalign = (e.key == BMADGPU_SBEND) ? (e.ref_tilt != 0 || offset) : (e.tilt != 0 || offset);
      double ds_step;
      int num_steps;
      resolve_steps(e, p, tilt_tot, &ds_step, &num_steps);
      out.ds_step[i] = ds_step;
      turn_ref += e.delta_ref_time;

      EleHdr h;
      std::memset(&h, 0, sizeof(h));
      h.n_step = 1;
      uint16_t flags = 0;
      std::vector<double> blk;
      int key = e.key;
      if (!e.is_on && key != BMADGPU_SBEND && key != BMADGPU_MULTIPOLE && key != BMADGPU_AB_MULTIPOLE)
        key = BMADGPU_DRIFT;  // track1_bmad.f90:51-60
      if (e.l == 0) flags |= F_ZERO_LEN;

      // aperture (check_aperture_limit.f90), offset_moves_aperture = F
      if (p.aperture_limit_on && e.aperture_at != BMADGPU_NO_END) {
        ApRec r;
        std::memset(&r, 0, sizeof(r));
        r.x1_lim = -e.x1_limit;
        r.x2_lim = e.x2_limit;
        r.y1_lim = -e.y1_limit;
        r.y2_lim = e.y2_limit;
        bool any = (r.x1_lim != 0 || r.x2_lim != 0 || r.y1_lim != 0 || r.y2_lim != 0);
        if (e.aperture_type == BMADGPU_APERTURE_ELLIPTICAL) {
          // elliptical_params_setup (check_aperture_limit.f90:361-387): limits set on one side
          // only skip the check; otherwise half width (max_aperture_limit for none) and centre
          auto setup = [&](double lim1, double lim2, double* w, double* c) {
            if ((lim1 == 0 && lim2 != 0) || (lim1 != 0 && lim2 == 0)) return false;
            *w = (lim2 - lim1) / 2;
            *c = (lim2 + lim1) / 2;
            if (*w == 0) *w = p.max_aperture_limit;
            *w = std::max(*w, 0.0);
            return true;
          };
          double xw, x0, yw, y0;
          if (setup(r.x1_lim, r.x2_lim, &xw, &x0) && setup(r.y1_lim, r.y2_lim, &yw, &y0)) {
            r.x1_lim = xw;
            r.x2_lim = x0;
            r.y1_lim = yw;
            r.y2_lim = y0;
            any = true;
            flags |= F_AP_ELLIPTICAL;
          } else {
            any = false;
          }
        }
        const bool coll = e.key == BMADGPU_ECOLLIMATOR || e.key == BMADGPU_RCOLLIMATOR;
        if (coll) {
          const double w[8] = {e.px_aperture_width2, e.px_aperture_center, e.py_aperture_width2,
                                e.py_aperture_center, e.z_aperture_width2, e.z_aperture_center,
                                e.pz_aperture_width2, e.pz_aperture_center};
          if (w[0] != 0 || w[2] != 0 || w[4] != 0 || w[6] != 0) {
            std::memcpy(r.win, w, sizeof(w));
            r.win_kind = e.key == BMADGPU_ECOLLIMATOR ? 1 : 2;
            flags |= F_AP_WINDOW;
            any = true;
          }
        }
        if (any) {
          h.ap_index = pk.add_ap(r);
          if (e.aperture_at == BMADGPU_ENTRANCE_END || e.aperture_at == BMADGPU_BOTH_ENDS) flags |= F_AP_ENTRANCE;
          if (e.aperture_at == BMADGPU_EXIT_END || e.aperture_at == BMADGPU_BOTH_ENDS) flags |= F_AP_EXIT;
        } else {
          flags &= (uint16_t)~(F_AP_ELLIPTICAL | F_AP_WINDOW);
        }
      }

      double a[kNPole], b[kNPole], ae[kNPole], be[kNPole];
      int ix_mag_max;
      const int ix_elec_max = elec_ab(e, ae, be);
      std::vector<double> mis, eblk;
      auto misalign_block = [&](double tilt) {
        mis = {e.x_offset, e.y_offset, l_cos(tilt), l_sin(tilt)};
        flags |= F_MISALIGN;
        if (pitched) {
          // offset_particle.f90:239-245, 279-282 (set) and 437-443, 477-480 (unset), straight
          // geometry: the offsets, the rotation floor_angles_to_w_mat(x_pitch, y_pitch, 0)
          // (bmad/geometry/floor_angles_to_w_mat.f90) and its inverse, the drift to the edge
          const double L_half = 0.5 * e.l;
          mis.insert(mis.end(), {e.z_offset, L_half, L_half - 0.0, L_half - e.l, (1 + 1) * L_half});
          const double s_the = l_sin(e.x_pitch), c_the = l_cos(e.x_pitch);
          const double s_phi = l_sin(e.y_pitch), c_phi = l_cos(e.y_pitch);
          const double s_psi = l_sin(0.0), c_psi = l_cos(0.0);
          const double winv[9] = {c_the * c_psi - s_the * s_phi * s_psi, c_phi * s_psi,
                                  -s_the * c_psi - c_the * s_phi * s_psi, -c_the * s_psi - s_the * s_phi * c_psi,
                                  c_phi * c_psi, s_the * s_psi - c_the * s_phi * c_psi,
                                  s_the * c_phi, s_phi, c_the * c_phi};
          const double w[9] = {c_the * c_psi - s_the * s_phi * s_psi, -c_the * s_psi - s_the * s_phi * c_psi,
                               s_the * c_phi, c_phi * s_psi, c_phi * c_psi, s_phi,
                               -s_the * c_psi - c_the * s_phi * s_psi, s_the * s_psi - c_the * s_phi * c_psi,
                               c_the * c_phi};
          mis.insert(mis.end(), winv, winv + 9);
          mis.insert(mis.end(), w, w + 9);
          flags |= F_PITCH;
        }
      };

      switch (key) {
        case BMADGPU_MARKER:
          h.kind = K_MARKER;
          break;
        case BMADGPU_DRIFT:
          h.kind = K_DRIFT;
          blk = {e.l};
          break;
        case BMADGPU_QUADRUPOLE: {  // track_a_quadrupole.f90
          h.kind = K_QUAD;
          mag_ab(e, tilt_tot, 0, a, b, &ix_mag_max);
          double b1 = pull_b1(a, b, &ix_mag_max);
          int n_step = 1;
          if (ix_mag_max > -1 || ix_elec_max > -1) n_step = std::max(nint(std::fabs(e.l) / ds_step), 1);
          double r_step = 1.0 / n_step;
          double step_len = e.l * r_step;
          blk = {b1, e.l, step_len};
          eblk = extra_block(e, p, ae, be, ix_elec_max, step_len / 2, step_len);
          if (ix_mag_max > -1) {
            flags |= F_KICKS;
            h.n_pole = (uint8_t)(ix_mag_max + 1);
            push_kicks(blk, a, b, ix_mag_max + 1, r_step / 2);
            push_kicks(blk, a, b, ix_mag_max + 1, r_step);
            if (kicks_b_from2(blk, 3, ix_mag_max + 1)) flags |= F_KICK_B_FROM2;
          }
          h.n_step = (uint16_t)(e.l == 0 ? 0 : n_step);
          if (has_misalign) misalign_block(tilt_tot);
          break;
        }
        case BMADGPU_SEXTUPOLE: case BMADGPU_OCTUPOLE: case BMADGPU_THICK_MULTIPOLE:
        case BMADGPU_MONITOR: case BMADGPU_INSTRUMENT: case BMADGPU_PIPE:
        case BMADGPU_RCOLLIMATOR: case BMADGPU_ECOLLIMATOR:
        case BMADGPU_KICKER: case BMADGPU_HKICKER: case BMADGPU_VKICKER:
        case BMADGPU_ELSEPARATOR: {  // track_a_thick_multipole.f90
          h.kind = K_THICK;
          mag_ab(e, tilt_tot, 0, a, b, &ix_mag_max);
          // the separator's field, :49-65: kick = |(hk, vk)| (charge sign), angle atan2(vk, hk)
          double sep_kick = 0, sep_angle = 0;
          if (key == BMADGPU_ELSEPARATOR) {
            const double rtc = 1.0 * (p.charge < 0 ? -1.0 : 1.0);
            const double hk = e.hkick * rtc, vk = e.vkick * rtc;
            sep_kick = std::sqrt(hk * hk + vk * vk);
            sep_angle = l_atan2(vk, hk);
          }
          int n_step = (sep_kick == 0 && ix_mag_max == -1 && ix_elec_max == -1)
                           ? 1 : std::max(nint(std::fabs(e.l / ds_step)), 1);
          double r_step = 1.0 / n_step;
          double step_len = e.l / n_step;
          blk = {step_len};
          if (key != BMADGPU_MONITOR && key != BMADGPU_INSTRUMENT && key != BMADGPU_PIPE &&
              key != BMADGPU_RCOLLIMATOR && key != BMADGPU_ECOLLIMATOR && key != BMADGPU_KICKER &&
              key != BMADGPU_HKICKER && key != BMADGPU_VKICKER)
            eblk = extra_block(e, p, ae, be, ix_elec_max, 1 * step_len / 2, 1 * step_len);
          if (key == BMADGPU_ELSEPARATOR) {
            eblk = extra_block(e, p, ae, be, ix_elec_max, 1 * step_len / 2, 1 * step_len);
            const double mr = p.mass / p.p0c;
            eblk[21] = sep_kick != 0 ? 1.0 : 0.0;
            eblk[22] = l_cos(sep_angle);
            eblk[23] = l_sin(sep_angle);
            eblk[24] = sep_angle != 0 ? 1.0 : 0.0;
            eblk[25] = (e.l == 0) ? 1.0 : sep_kick / e.l;
            eblk[26] = p.p0c / p.e_tot;
            eblk[27] = mr * mr;
          }
          if (ix_mag_max > -1) {
            flags |= F_KICKS;
            h.n_pole = (uint8_t)(ix_mag_max + 1);
            push_kicks(blk, a, b, ix_mag_max + 1, r_step / 2);
            push_kicks(blk, a, b, ix_mag_max + 1, r_step);
            if (kicks_b_from2(blk, 1, ix_mag_max + 1)) flags |= F_KICK_B_FROM2;
          }
          h.n_step = (uint16_t)n_step;
          if (has_misalign) misalign_block(tilt_tot);
          break;
        }
        case BMADGPU_SBEND: {  // track_a_bend.f90
          h.kind = K_SBEND;
          mag_ab(e, 0, e.ref_tilt, a, b, &ix_mag_max);
          double b1 = pull_b1(a, b, &ix_mag_max);
          if (std::fabs(b1) < 1e-10) {
            b[1] = b1;
            b1 = 0;
          }
          double g = e.g, dg;
          if (e.l == 0) {
            dg = 0;
          } else {
            dg = b[0] / e.l;
            b[0] = 0;
          }
          double g_tot = g + dg;
          if (!e.is_on) {
            dg = -g;
            g_tot = 0;
            b1 = 0;
          }
          int n_step = 1;
          if (ix_mag_max > -1 || ix_elec_max > -1) n_step = std::max(nint(std::fabs(e.l) / ds_step), 1);
          double r_step = 1.0 / n_step;
          double step_len = e.l / n_step;
          double angle = g * step_len;
          eblk = extra_block(e, p, ae, be, ix_elec_max, step_len * 0.5, step_len * 1.0);
          double gl = g * step_len;
          blk = {step_len, g, g_tot, dg, angle, l_cos(angle), l_sin(angle), sinc0(angle), cosc0(angle),
                 (gl * gl) * sincc0(angle), (b1 != 0 && e.l != 0) ? b1 / e.l : 0.0,
                 r_step * p.p0c / (2.99792458e8 * p.charge)};
          if (b1 != 0) flags |= F_BEND_K1;
          else if ((g == 0 && dg == 0) || step_len == 0) flags |= F_BEND_DRIFT;
          // Hwang edge coefficients (fringe_mod.f90:262-290); bend_edge_kick acts for
          // fringe_type basic_bend / hard_edge_only when at_this_ele_end(fringe_at).
          double ge = e.is_on ? (e.g + e.dg) : 0.0;
          double k1e = e.is_on ? e.k1 : 0.0;
          for (int end = 0; end < 2; end++) {
            double ee = end == 0 ? e.e1 : e.e2;
            double fint_gap = end == 0 ? e.fint * e.hgap : e.fintx * e.hgapx;
            if (e.fringe_type == BMADGPU_FRINGE_HARD_EDGE_ONLY || e.fringe_type == BMADGPU_FRINGE_SAD_FULL) fint_gap = 0;
            double cos_e = l_cos(ee), sin_e = l_sin(ee);
            double tan_e = sin_e / cos_e, sec_e = 1 / cos_e;
            double gt = ge * tan_e;
            double gt2 = ge * (tan_e * tan_e);
            double gs2 = ge * (sec_e * sec_e);
            double k1_tane = k1e * tan_e * 1.0;
            double fg_factor = 2 * fint_gap * gs2 * ge * sec_e * (1 + sin_e * sin_e);
            double cdpx = gt * ge * (1 + 2 * (tan_e * tan_e));
            blk.insert(blk.end(), {gt, gt2, gs2, k1_tane, fg_factor, ge, cdpx});
          }
          if (e.fringe_type == BMADGPU_FRINGE_BASIC_BEND || e.fringe_type == BMADGPU_FRINGE_HARD_EDGE_ONLY) {
            if (e.fringe_at == BMADGPU_ENTRANCE_END || e.fringe_at == BMADGPU_BOTH_ENDS) flags |= F_EDGE_IN;
            if (e.fringe_at == BMADGPU_EXIT_END || e.fringe_at == BMADGPU_BOTH_ENDS) flags |= F_EDGE_OUT;
          } else if (e.fringe_type != BMADGPU_FRINGE_NONE && e.fringe_type != BMADGPU_FRINGE_FULL) {
            fail(BMADGPU_EUNSUPPORTED, "sbend fringe_type other than none/basic_bend/hard_edge_only/full");
          }
          if (ix_mag_max > -1) {
            flags |= F_KICKS;
            h.n_pole = (uint8_t)(ix_mag_max + 1);
            push_kicks(blk, a, b, ix_mag_max + 1, 1.0);
          }
          h.n_step = (uint16_t)n_step;
          if (offset) {  // offsets, pitches or z_offset: the bend frame
            mis = bend_frame_block(e);
            flags |= F_MISALIGN | F_PITCH;
          } else if (has_misalign) {  // ref_tilt only: tilt_coords
            mis = {0.0, 0.0, l_cos(e.ref_tilt), l_sin(e.ref_tilt)};
            flags |= F_MISALIGN;
          }
          break;
        }
        case BMADGPU_MULTIPOLE: case BMADGPU_AB_MULTIPOLE: {  // track1_bmad.f90:142-166
          h.kind = K_THIN;
          double knl[kNPole], tn[kNPole];
          for (int n = 0; n < kNPole; n++) { knl[n] = 0; tn[n] = 0; }
          if (key == BMADGPU_MULTIPOLE) {
            // multipole_ele_to_kt.f90: knl = knl_pole, tilt = tilt_pole + tilt_tot
            for (int n = 0; n < kNPole; n++) { knl[n] = e.a_pole[n]; tn[n] = e.b_pole[n] + tilt_tot; }
            if (e.a_pole[0] != 0) flags |= F_REF_ORB_N0;
          } else {
            // multipole_ele_to_ab(use_ele_tilt = T) then multipole_ab_to_kt
            mag_ab(e, tilt_tot, 0, a, b, &ix_mag_max);
            tilt_ab(tilt_tot, a, b, ix_mag_max);
            if (ix_mag_max > -1)
              for (int n = 0; n < kNPole; n++) ab_to_kt(a[n], b[n], n, &knl[n], &tn[n]);
          }
          int top = -1;
          for (int n = 0; n < kNPole; n++)
            if (knl[n] != 0) top = n;
          blk.clear();
          for (int n = 0; n <= top; n++) {
            bool tz = (tn[n] == 0);
            blk.insert(blk.end(), {knl[n], tz ? 1.0 : l_cos(tn[n]), tz ? 0.0 : l_sin(tn[n]), tz ? 1.0 : 0.0});
          }
          if (top >= 0) flags |= F_KICKS;
          h.n_pole = (uint8_t)(top + 1);
          if (e.x_offset != 0 || e.y_offset != 0) {
            mis = {e.x_offset, e.y_offset, 1.0, 0.0};  // offset_particle with set_tilt = .false.
            flags |= F_MISALIGN;
          }
          break;
        }
        case BMADGPU_RFCAVITY: {  // track_a_rfcavity.f90
          h.kind = K_RFCAV;
          if (e.rf_frequency == 0 && e.voltage != 0) fail(BMADGPU_EINVAL, "rfcavity with zero rf_frequency");
          mag_ab(e, tilt_tot, 0, a, b, &ix_mag_max);
          int n_slice = std::max(1, nint(std::fabs(e.l) / ds_step));
          double voltage = (e.is_on ? e.voltage : 0.0) * 1.0;
          blk = {voltage, e.rf_frequency, e.phi0, 2 * kPi * e.phi0_multipass, e.l / n_slice, (double)n_slice};
          if (ix_mag_max > -1) {
            flags |= F_KICKS;
            h.n_pole = (uint8_t)(ix_mag_max + 1);
            push_kicks(blk, a, b, ix_mag_max + 1, 0.5 * 1.0);
          }
          h.n_step = (uint16_t)std::min(n_slice, 65535);
          if (n_slice > 65535) fail(BMADGPU_EUNSUPPORTED, "too many rf slices");
          if (e.tilt != 0 || e.x_offset != 0 || e.y_offset != 0 || pitched) misalign_block(tilt_tot);
          break;
        }
        default:
          fail(BMADGPU_EUNSUPPORTED, "element type");
      }
      if ((flags & F_MISALIGN) && h.kind != K_SBEND && mis.size() >= 4 && mis[3] != 0) flags |= F_TILT;
      blk.insert(blk.end(), mis.begin(), mis.end());
      if (!eblk.empty() && (h.kind == K_QUAD || h.kind == K_THICK || h.kind == K_SBEND)) {
        flags |= F_EXTRA;
        h.extra = pk.add_block(eblk);
      }
      h.flags = flags;
      h.param = pk.add_block(blk);
      out.n_step[i] = h.n_step;
      pk.hdr.push_back(h);
    }
    if (pk.ap.size() > 0xFFFF) throw Fail{BMADGPU_EUNSUPPORTED, "too many distinct apertures"};
    if (pk.pool.empty()) pk.pool.push_back(0.0);
    TableInfo& ti = out.info;
    ti.n_ele = (uint32_t)n_ele;
    ti.n_ap = (uint32_t)pk.ap.size();
    ti.hdr_bytes = (uint32_t)(n_ele * sizeof(EleHdr));
    ti.ap_bytes = (uint32_t)(pk.ap.size() * sizeof(ApRec));
    ti.pool_doubles = (uint32_t)pk.pool.size();
    size_t total = ti.hdr_bytes + ti.ap_bytes + pk.pool.size() * sizeof(double);
    total = (total + 15) & ~size_t(15);
    ti.total_bytes = (uint32_t)total;
    ti.turn_ref_time = turn_ref;
    ti.rare = 0;
    for (const EleHdr& h : pk.hdr)
      if (h.flags & (F_EXTRA | F_PITCH | F_AP_WINDOW)) ti.rare = 1;
    out.image.assign(total, 0);
    std::memcpy(out.image.data(), pk.hdr.data(), ti.hdr_bytes);
    if (ti.ap_bytes) std::memcpy(out.image.data() + ti.hdr_bytes, pk.ap.data(), ti.ap_bytes);
    std::memcpy(out.image.data() + ti.hdr_bytes + ti.ap_bytes, pk.pool.data(), pk.pool.size() * sizeof(double));
    out.ref_time_prefix.assign(n_ele + 1, 0.0);
    for (int i = 0; i < n_ele; i++) out.ref_time_prefix[i + 1] = out.ref_time_prefix[i] + eles[i].delta_ref_time;
    return BMADGPU_OK;
  } catch (const Fail& f) {
    err = f.msg;
    return f.code;
  }
}

}  // namespace bmadgpu
