// bmad_oracle.cpp -- CPU ORACLE, test infrastructure only (see bmad_oracle.h).
//
// A scalar restatement of Bmad's bmad_standard tracking of one charged particle through
// drift / quadrupole / sbend / sextupole / octupole / thick_multipole / multipole /
// ab_multipole / rfcavity / marker / monitor / instrument / pipe / ecollimator / rcollimator
// elements, with rectangular and elliptical apertures and the collimators' phase-space windows,
// and of the bunch loop around it. Every routine names the
// Fortran file and lines it restates (paths inside bmad-sim/bmad-ecosystem). Expressions keep
// the Fortran operand order; the file is compiled with -ffp-contract=off.
//
// Not restated (returns BMADGPU_EUNSUPPORTED): exact_multipoles, sbend fringe_type
// soft_edge_only / sad_full / linear_edge edges, ac_kickers, reversed
// orientation / direction / time, absolute time tracking, radiation and spin.

#include "bmad_oracle.h"

#include <quadmath.h>
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <algorithm>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef __float128 qp;

// The libm of the restated routines: the host's (default: glibc, as a gfortran build of the
// reference on Linux uses), or eight functions the caller installs with oracle_set_libm (the
// tests install correctly rounded ones to compare with the device, whose maps are correctly
// rounded). atan(v) is taken as atan2(v, 1), the same value.
double h_sin(double x) { return std::sin(x); }
double h_cos(double x) { return std::cos(x); }
double h_asin(double x) { return std::asin(x); }
double h_atan2(double y, double x) { return std::atan2(y, x); }
double h_sinh(double x) { return std::sinh(x); }
double h_cosh(double x) { return std::cosh(x); }
double h_exp(double x) { return std::exp(x); }
double h_tan(double x) { return std::tan(x); }
struct Libm {
  double (*sin)(double);
  double (*cos)(double);
  double (*asin)(double);
  double (*atan2)(double, double);
  double (*sinh)(double);
  double (*cosh)(double);
  double (*exp)(double);
  double (*tan)(double);
};
Libm lm = {h_sin, h_cos, h_asin, h_atan2, h_sinh, h_cosh, h_exp, h_tan};

// sim_utils/interfaces/physical_constants.f90:12-13, 34
const double pi = 3.141592653589793238462643383279;
const double twopi = 2 * pi;
const double c_light = 2.99792458e8;

enum { magnetic = 1, electric = 2 };
enum { first_track_edge = 11, second_track_edge = 12 };
enum { set_ = 1, unset_ = 0 };
const int n_pole_maxx = 21;

// ---------------------------------------------------------------------------------------------
// Special functions, sim_utils/special_functions/*.f90

// sinc.f90:15 (nd = 0 and nd = 1 branches)
double sinc(double x, int nd = 0) {
  const double c1 = -1.0 / 3.0, c2 = 1.0 / 30.0, c3 = -1.0 / 840.0, c4 = 1.0 / 45360.0;
  double x2 = x * x;
  if (nd == 0) {
    if (std::fabs(x) < 1e-8) return 1.0;
    return lm.sin(x) / x;
  }
  if (std::fabs(x) < 0.1) return x * (c1 + x2 * (c2 + x2 * (c3 + x2 * c4)));
  return (x * lm.cos(x) - lm.sin(x)) / x2;
}

// cosc.f90:15
double cosc(double x) {
  if (std::fabs(x) < 1e-8) return 0.50;
  double s = sinc(x / 2);
  return 0.5 * (s * s);
}

// sincc.f90:15
double sincc(double x) {
  const double c0 = 1.0 / 6.0, c1 = -1.0 / 120.0, c2 = 1.0 / 5040.0, c3 = -1.0 / 362880.0;
  double x2 = x * x;
  if (std::fabs(x) < 0.1) return c0 + x2 * (c1 + x2 * (c2 + x2 * c3));
  return (x - lm.sin(x)) / (x * x2);
}

// sqrt_one.f90:18
double sqrt_one(double x) {
  double sq = std::sqrt(1 + x);
  double rad = sq + 1;
  return x / rad;
}

// Fortran MODULO for reals: result has the sign of p, |result| < |p|.
double fmodulo(double a, double p) {
  double r = std::fmod(a, p);
  if (r != 0 && ((r < 0) != (p < 0))) r += p;
  return r;
}
qp qmodulo(qp a, qp p) {
  qp r = fmodq(a, p);
  if (r != 0 && ((r < 0) != (p < 0))) r += p;
  return r;
}

// modulo2_mod.f90:85-100 (modulo2_dp) and the qp twin
double modulo2(double x, double amp) {
  double mod2 = fmodulo(x, 2 * amp);
  if (mod2 >= amp) mod2 = mod2 - 2 * amp;
  return mod2;
}
qp modulo2q(qp x, qp amp) {
  qp mod2 = qmodulo(x, 2 * amp);
  if (mod2 >= amp) mod2 = mod2 - 2 * amp;
  return mod2;
}

// Fortran x**m for a run-time integer m (gfortran lowers it to libgcc's binary powering).
double powi(double x, int m) {
  unsigned n = m < 0 ? -m : m;
  double y = (n % 2) ? x : 1;
  while (n >>= 1) {
    x = x * x;
    if (n % 2) y = y * x;
  }
  return m < 0 ? 1 / y : y;
}

// mexp.f90:14-33
double mexp(double x, int m) {
  if (m < 0) return 0;
  if (m == 0) return 1;
  return powi(x, m);
}

// c_multi.f90:19-75: signed binomial / n! table; c_multi(n, m, no_n_fact=T) = c(n,m) * n!.
struct CMulti {
  double c[n_pole_maxx + 1][n_pole_maxx + 1];
  double nfact[n_pole_maxx + 1];
  CMulti() {
    std::memset(c, 0, sizeof(c));
    c[0][0] = 1;
    for (int in = 1; in <= n_pole_maxx; in++) {
      c[in][0] = 1;
      c[in][in] = 1;
      for (int im = 1; im <= in - 1; im++) c[in][im] = c[in - 1][im - 1] + c[in - 1][im];
    }
    nfact[0] = 1;
    for (int in = 0; in <= n_pole_maxx; in++) {
      if (in > 0) nfact[in] = in * nfact[in - 1];
      for (int im = 0; im <= in; im++) {
        c[in][im] = c[in][im] / nfact[in];
        if (im % 4 == 0) c[in][im] = -c[in][im];
        if (im % 4 == 3) c[in][im] = -c[in][im];
      }
    }
  }
  double no_n_fact(int n, int m) const { return c[n][m] * nfact[n]; }
};
const CMulti cm;

// sim_utils/special_functions/factorial.f90 (exact below 13!)
double factorial(int n) {
  static const double f[] = {1., 1., 2., 6., 24., 120., 720., 5040., 40320., 362880., 3628800.,
                             39916800., 479001600., 6.227020800000e+09, 8.717829120000e+10,
                             1.307674368000e+12, 2.092278988800e+13, 3.556874280960e+14,
                             6.402373705728e+15, 1.216451004088e+17, 2.432902008177e+18,
                             5.109094217171e+19};
  return f[n];
}

int nint(double x) { return (int)std::lround(x); }  // Fortran NINT: half away from zero

// sim_utils/math/max_nonzero.f90:19-44
int max_nonzero(const double* a, const double* b, int ub) {
  for (int i = ub; i >= 0; i--) {
    if (a[i] != 0) return i;
    if (b && b[i] != 0) return i;
  }
  return -1;
}

// ---------------------------------------------------------------------------------------------
// Particle and element state

struct Coord {
  double vec[6];
  double beta, p0c, s, phase1;
  qp t;
  int state, location, ix_ele;
};

struct Ele {
  const bmadgpu_element* e;
  const bmadgpu_param* p;
  int ix_ele;
  double tilt_tot, ref_tilt_tot;
  bool has_misalign;
  double ds_step;
  int num_steps;
  double s_start, s;
  bool has_elec;   // associated(ele%a_pole_elec)
  bool has_mag;    // associated(ele%a_pole)
};

// has_hkick_attributes (attribute_mod.f90:746-765, 1879) for the keys on the path
bool key_has_hkick(int key) {
  switch (key) {
    case BMADGPU_QUADRUPOLE: case BMADGPU_SBEND: case BMADGPU_SEXTUPOLE: case BMADGPU_OCTUPOLE:
    case BMADGPU_THICK_MULTIPOLE: case BMADGPU_RFCAVITY: case BMADGPU_MONITOR: case BMADGPU_INSTRUMENT:
    case BMADGPU_RCOLLIMATOR: case BMADGPU_ECOLLIMATOR: case BMADGPU_KICKER: case BMADGPU_ELSEPARATOR:
      return true;
  }
  return false;
}

bool key_has_orientation(int key) {
  switch (key) {
    case BMADGPU_MARKER: return false;
  }
  return true;
}

// ---------------------------------------------------------------------------------------------
// multipole_ele_to_ab, bmad/code/multipole_ele_to_ab.f90:31-678 (non-slave elements)

// tilt_this_multipole, :440-467
void tilt_this_multipole(const Ele& ele, int sgn, double* a, double* b, int ix_pole_max) {
  double tilt = (ele.e->key == BMADGPU_SBEND) ? sgn * ele.ref_tilt_tot : sgn * ele.tilt_tot;
  if (tilt == 0) return;
  for (int n = 0; n <= ix_pole_max; n++) {
    if (a[n] == 0 && b[n] == 0) continue;
    double an = a[n], bn = b[n];
    double cos_t = lm.cos((n + 1) * tilt);
    double sin_t = lm.sin((n + 1) * tilt);
    b[n] = bn * cos_t + an * sin_t;
    a[n] = -bn * sin_t + an * cos_t;
  }
}

// multipole1_kt_to_ab, bmad/low_level/multipole1_kt_to_ab.f90 (knsl = 0)
void multipole1_kt_to_ab(double knl, double tn, int n, double* an, double* bn) {
  if (knl == 0) { *an = 0; *bn = 0; return; }
  double angle = -tn * (n + 1);
  *bn = (knl * lm.cos(angle) - 0.0 * lm.sin(angle)) / factorial(n);
  *an = (knl * lm.sin(angle) + 0.0 * lm.cos(angle)) / factorial(n);
}

// multipole1_ab_to_kt, bmad/low_level/multipole1_ab_to_kt.f90:17
void multipole1_ab_to_kt(double an, double bn, int n, double* knl, double* tn) {
  if (an == 0 && bn == 0) { *knl = 0; *tn = 0; return; }
  double a = an, b = bn;
  *knl = factorial(n) * std::sqrt(a * a + b * b);
  *tn = -lm.atan2(a, b) / (n + 1);
  if (2 * (n + 1) * std::fabs(*tn) > pi) {
    *knl = -*knl;
    double sgn = (*tn < 0) ? -1.0 : 1.0;
    *tn = sgn * (std::fabs(*tn) - pi / (n + 1));
  }
}

// convert_this_ab, :472-600 (this_ele == ele, so the relative tilt is 0)
int convert_this_ab(const Ele& ele, int p_type, const double* a_pole, const double* b_pole,
                    double* this_a, double* this_b) {
  const bmadgpu_element* e = ele.e;
  for (int i = 0; i <= n_pole_maxx; i++) { this_a[i] = a_pole[i]; this_b[i] = b_pole[i]; }
  int ix_max = max_nonzero(this_a, this_b, n_pole_maxx);
  if (ix_max < 0) return 0;
  if (e->field_master) return BMADGPU_EUNSUPPORTED;
  if (!e->scale_multipoles) return 0;
  if (p_type == electric) {
    double radius = e->r0_elec;
    if (radius != 0 && radius != 1) {
      double factor = radius;
      for (int n = 0; n <= n_pole_maxx; n++) {
        factor = factor / radius;
        this_a[n] = factor * this_a[n];
        this_b[n] = factor * this_b[n];
      }
    }
    return 0;
  }
  double cnst;
  int ref_exp;
  switch (e->key) {
    case BMADGPU_SBEND: cnst = e->l * (e->g + e->dg); ref_exp = 0; break;
    case BMADGPU_QUADRUPOLE: cnst = e->k1 * e->l; ref_exp = 1; break;
    case BMADGPU_SEXTUPOLE: cnst = e->k2 * e->l; ref_exp = 2; break;
    case BMADGPU_OCTUPOLE: cnst = e->k3 * e->l; ref_exp = 3; break;
    case BMADGPU_KICKER: case BMADGPU_ELSEPARATOR:
      if (e->hkick == 0) cnst = e->vkick;
      else if (e->vkick == 0) cnst = e->hkick;
      else cnst = std::sqrt(e->hkick * e->hkick + e->vkick * e->vkick);
      ref_exp = 0;
      break;
    case BMADGPU_HKICKER: case BMADGPU_VKICKER: cnst = e->kick; ref_exp = 0; break;
    case BMADGPU_AB_MULTIPOLE: case BMADGPU_THICK_MULTIPOLE: case BMADGPU_RFCAVITY: return 0;
    default: return BMADGPU_EUNSUPPORTED;
  }
  double radius = e->r0_mag;
  if (radius == 0) {
    for (int n = 0; n <= n_pole_maxx; n++) { this_a[n] = cnst * this_a[n]; this_b[n] = cnst * this_b[n]; }
  } else {
    double factor = cnst * powi(radius, ref_exp + 1);
    for (int n = 0; n <= n_pole_maxx; n++) {
      factor = factor / radius;
      this_a[n] = factor * this_a[n];
      this_b[n] = factor * this_b[n];
    }
  }
  return 0;
}

// this_ele_non_multipoles, :326-405
void this_ele_non_multipoles(const Ele& ele, int p_type, double a_kick[4], double b_kick[4]) {
  const bmadgpu_element* e = ele.e;
  for (int i = 0; i < 4; i++) { a_kick[i] = 0; b_kick[i] = 0; }
  if (p_type != magnetic) return;
  switch (e->key) {  // multipole_ele_to_ab.f90:339-346
    case BMADGPU_HKICKER: b_kick[0] = -e->kick; return;
    case BMADGPU_VKICKER: a_kick[0] = e->kick; return;
    case BMADGPU_KICKER:
      b_kick[0] = -e->hkick;
      a_kick[0] = e->vkick;
      return;
    case BMADGPU_ELSEPARATOR: return;
  }
  double hk = e->hkick, vk = e->vkick;
  if (key_has_hkick(e->key) && (hk != 0 || vk != 0)) {
    double tilt = (e->key == BMADGPU_SBEND) ? ele.ref_tilt_tot : ele.tilt_tot;
    if (tilt != 0) {
      double cos_t = lm.cos(tilt), sin_t = lm.sin(tilt);
      b_kick[0] = -hk * cos_t - vk * sin_t;
      a_kick[0] = -hk * sin_t + vk * cos_t;
    } else {
      b_kick[0] = -hk;
      a_kick[0] = vk;
    }
  }
  switch (e->key) {
    case BMADGPU_QUADRUPOLE: b_kick[1] = e->k1 * e->l; break;
    case BMADGPU_SBEND:
      b_kick[0] = b_kick[0] + e->dg * e->l;
      b_kick[1] = e->k1 * e->l;
      b_kick[2] = e->k2 * e->l / 2.0;
      break;
    case BMADGPU_SEXTUPOLE: b_kick[2] = e->k2 * e->l / 2.0; break;
    case BMADGPU_OCTUPOLE: b_kick[3] = e->k3 * e->l / 6.0; break;
  }
}

// pull_this_b1, :664-676
double pull_this_b1(double* a, double* b, int* ix_pole_max) {
  double b1 = b[1];
  b[1] = 0;
  if (*ix_pole_max > 1) return b1;
  *ix_pole_max = max_nonzero(a, b, 1);
  return b1;
}

int multipole_ele_to_ab(const Ele& ele, bool use_ele_tilt, int* ix_pole_max, double* a, double* b,
                        int pole_type, bool include_kicks, double* b1) {
  const bmadgpu_element* e = ele.e;
  *ix_pole_max = -1;
  for (int i = 0; i <= n_pole_maxx; i++) { a[i] = 0; b[i] = 0; }
  if (b1) *b1 = 0;
  if (!e->is_on || e->key == BMADGPU_PIPE) return 0;

  if (e->key == BMADGPU_MULTIPOLE) {  // :88-112
    if (pole_type == electric || !ele.has_mag) return 0;
    for (int n = 0; n <= n_pole_maxx; n++) multipole1_kt_to_ab(e->a_pole[n], e->b_pole[n], n, &a[n], &b[n]);
    *ix_pole_max = max_nonzero(a, b, n_pole_maxx);
    if (b1) *b1 = pull_this_b1(a, b, ix_pole_max);
    return 0;
  }

  const double* a_pole = (pole_type == electric) ? e->a_pole_elec : e->a_pole;
  const double* b_pole = (pole_type == electric) ? e->b_pole_elec : e->b_pole;
  bool assoc = (pole_type == electric) ? ele.has_elec : ele.has_mag;
  if (assoc) {
    int err = convert_this_ab(ele, pole_type, a_pole, b_pole, a, b);
    if (err) return err;
  }
  double a_kick[4], b_kick[4];
  this_ele_non_multipoles(ele, pole_type, a_kick, b_kick);
  if (include_kicks) {
    for (int i = 0; i < 4; i++) { a[i] = a[i] + a_kick[i]; b[i] = b[i] + b_kick[i]; }
  }
  *ix_pole_max = max_nonzero(a, b, n_pole_maxx);
  if (use_ele_tilt) tilt_this_multipole(ele, +1, a, b, *ix_pole_max);
  if (b1) *b1 = pull_this_b1(a, b, ix_pole_max);
  return 0;
}

// multipole_ele_to_kt, bmad/code/multipole_ele_to_kt.f90
int multipole_ele_to_kt(const Ele& ele, bool use_ele_tilt, int* ix_pole_max, double* knl, double* tilt,
                        int pole_type, bool include_kicks) {
  const bmadgpu_element* e = ele.e;
  if (e->key == BMADGPU_MULTIPOLE) {
    if (pole_type == electric) {
      for (int i = 0; i <= n_pole_maxx; i++) { knl[i] = 0; tilt[i] = 0; }
      *ix_pole_max = 0;
      return 0;
    }
    for (int i = 0; i <= n_pole_maxx; i++) { knl[i] = e->a_pole[i]; tilt[i] = e->b_pole[i] + ele.tilt_tot; }
    *ix_pole_max = max_nonzero(knl, nullptr, n_pole_maxx);
    return 0;
  }
  double a[n_pole_maxx + 1], b[n_pole_maxx + 1];
  int err = multipole_ele_to_ab(ele, use_ele_tilt, ix_pole_max, a, b, pole_type, include_kicks, nullptr);
  if (err) return err;
  if (*ix_pole_max > -1) {
    for (int n = 0; n <= n_pole_maxx; n++) multipole1_ab_to_kt(a[n], b[n], n, &knl[n], &tilt[n]);
  } else {
    for (int i = 0; i <= n_pole_maxx; i++) { knl[i] = 0; tilt[i] = 0; }
  }
  return 0;
}

// ---------------------------------------------------------------------------------------------
// Multipole kicks, bmad/modules/multipole_mod.f90

// ab_multipole_kick, :314-401 (ele_orientation = 0 ignores orientation and species)
void ab_multipole_kick(double a, double b, int n, int ele_orientation, const Coord& coord,
                       const bmadgpu_param* p, double* kx, double* ky, int pole_type, double scale,
                       bool has_scale) {
  *kx = 0;
  *ky = 0;
  if (a == 0 && b == 0) return;
  double a2, b2, f;
  if (pole_type == electric) {
    f = p->charge / (coord.beta * coord.p0c);
    a2 = a * f;
    b2 = -b * f;
  } else {
    if (ele_orientation == 0) {
      a2 = a;
      b2 = b;
    } else {
      f = 1.0;  // direction * orientation * charge_to_mass_of(species)/charge_to_mass_of(ref_species)
      a2 = a * f;
      b2 = b * f;
    }
  }
  if (has_scale) {
    a2 = scale * a2;
    b2 = scale * b2;
  }
  double x = coord.vec[0], y = coord.vec[2];
  for (int m = 0; m <= n; m += 2) {
    f = cm.no_n_fact(n, m) * mexp(x, n - m) * mexp(y, m);
    *kx = *kx + b2 * f;
    *ky = *ky - a2 * f;
  }
  for (int m = 1; m <= n; m += 2) {
    f = cm.no_n_fact(n, m) * mexp(x, n - m) * mexp(y, m);
    *kx = *kx + a2 * f;
    *ky = *ky + b2 * f;
  }
}

// ab_multipole_kicks, :82-174
void ab_multipole_kicks(const double* an, const double* bn, int ix_pole_max, const Ele& ele, Coord& orbit,
                        int pole_type, double scale) {
  double kx_tot = 0, ky_tot = 0;
  Coord orb0 = orbit;
  double r = ele.p->p0c / orbit.p0c;
  for (int n = 0; n <= ix_pole_max; n++) {
    double kx, ky;
    ab_multipole_kick(r * an[n], r * bn[n], n, 1, orbit, ele.p, &kx, &ky, pole_type, scale, true);
    kx_tot = kx_tot + kx;
    ky_tot = ky_tot + ky;
  }
  orbit.vec[1] = orbit.vec[1] + kx_tot;
  orbit.vec[3] = orbit.vec[3] + ky_tot;
  if (pole_type == magnetic) return;
  // Electric: energy change, :129-141
  double rp0 = 1 + orb0.vec[5];
  double alpha = (kx_tot * (2 * orb0.vec[1] + kx_tot) + ky_tot * (2 * orb0.vec[3] + ky_tot)) / (rp0 * rp0);
  if (alpha < -1) {
    orbit.state = BMADGPU_LOST_PZ;
    return;
  }
  double dpz = (1 + orb0.vec[5]) * sqrt_one(alpha);
  orbit.vec[5] = orb0.vec[5] + dpz;
  double rp1 = 1 + orbit.vec[5];
  double mp = ele.p->mass / orbit.p0c;
  orbit.beta = (1 + orbit.vec[5]) / std::sqrt(rp1 * rp1 + mp * mp);
  orbit.vec[4] = orb0.vec[4] * orbit.beta / orb0.beta;
}

// multipole_kick, :203-286 (magnetic)
void multipole_kick(double knl, double tilt, int n, Coord& coord, bool ref_orb_offset) {
  if (knl == 0) return;
  double t = tilt;
  double charge = 1.0;  // direction * time_dir * orientation * (q/m)/(q/m)_ref
  double sin_ang, cos_ang, x, y;
  if (t == 0) {
    sin_ang = 0;
    cos_ang = 1;
    x = coord.vec[0];
    y = coord.vec[2];
  } else {
    sin_ang = lm.sin(t);
    cos_ang = lm.cos(t);
    x = coord.vec[0] * cos_ang + coord.vec[2] * sin_ang;
    y = -coord.vec[0] * sin_ang + coord.vec[2] * cos_ang;
  }
  if (n == 0 && ref_orb_offset) {
    coord.vec[1] = coord.vec[1] + charge * knl * cos_ang * coord.vec[5];
    coord.vec[3] = coord.vec[3] + charge * knl * sin_ang * coord.vec[5];
    coord.vec[4] = coord.vec[4] - charge * knl * (cos_ang * coord.vec[0] + sin_ang * coord.vec[2]);
    return;
  }
  double x_terms[n_pole_maxx + 1], y_terms[n_pole_maxx + 1];
  x_terms[n] = 1.0;
  y_terms[0] = 1.0;
  for (int m = 1; m <= n; m++) {
    x_terms[n - m] = x_terms[n - m + 1] * x;
    y_terms[m] = y_terms[m - 1] * y;
  }
  double x_value = 0, y_value = 0;
  for (int m = 0; m <= n; m += 2) x_value = x_value + cm.c[n][m] * x_terms[m] * y_terms[m];
  for (int m = 1; m <= n; m += 2) y_value = y_value + cm.c[n][m] * x_terms[m] * y_terms[m];
  double x_vel = charge * knl * x_value;
  double y_vel = charge * knl * y_value;
  if (t == 0) {
    coord.vec[1] = coord.vec[1] + x_vel;
    coord.vec[3] = coord.vec[3] + y_vel;
  } else {
    coord.vec[1] = coord.vec[1] + x_vel * cos_ang - y_vel * sin_ang;
    coord.vec[3] = coord.vec[3] + x_vel * sin_ang + y_vel * cos_ang;
  }
}

// ---------------------------------------------------------------------------------------------
// Drift, bmad/low_level/track_a_drift.f90:25-116 (orb%direction = +1)
void track_a_drift(Coord& orb, double length, const bmadgpu_param* p, bool include_ref_motion = true,
                   int ele_orientation = 1) {
  if (length == 0) return;
  double delta = orb.vec[5];
  double rel_pc = 1 + delta;
  int rel_z_vel = ele_orientation * 1;
  double px_rel = rel_z_vel * orb.vec[1] / rel_pc;
  double py_rel = rel_z_vel * orb.vec[3] / rel_pc;
  double pxy2 = px_rel * px_rel + py_rel * py_rel;
  if (pxy2 >= 1) {
    orb.state = BMADGPU_LOST_PZ;
    return;
  }
  double ps_rel = std::sqrt(1 - pxy2);
  orb.vec[0] = orb.vec[0] + length * px_rel / ps_rel;
  orb.vec[2] = orb.vec[2] + length * py_rel / ps_rel;
  double dz;
  if (orb.beta > 0) {
    if (include_ref_motion) {
      double mc2 = p->mass;
      double pr = orb.p0c * rel_pc;
      dz = length * (sqrt_one((mc2 * mc2 * (2 * delta + delta * delta)) / (pr * pr + mc2 * mc2)) +
                     sqrt_one(-pxy2) / ps_rel);
      orb.s = orb.s + 1 * length;
    } else {
      dz = -length / ps_rel;
    }
    double dt = rel_z_vel * length / (orb.beta * ps_rel * c_light);
    orb.t = orb.t + (qp)dt;
  } else {
    if (include_ref_motion) {
      dz = length * (1 - 1 / ps_rel);
      orb.s = orb.s + length;
    } else {
      dz = -length / ps_rel;
    }
  }
  orb.vec[4] = orb.vec[4] + rel_z_vel * dz;
}

// quad_mat2_calc, bmad/low_level/quad_mat2_calc.f90:22-81 (no dz_dpz_coef)
void quad_mat2_calc(double k1, double length, double rel_p, double mat2[2][2], double zc[3]) {
  double sqrt_k = std::sqrt(std::fabs(k1));
  double sk_l = sqrt_k * length;
  double cx, sx;
  if (std::fabs(sk_l) < 1e-10) {
    double k_l2 = k1 * (length * length);
    cx = 1 + k_l2 / 2;
    sx = (1 + k_l2 / 6) * length;
  } else if (k1 < 0) {
    cx = lm.cos(sk_l);
    sx = lm.sin(sk_l) / sqrt_k;
  } else {
    cx = lm.cosh(sk_l);
    sx = lm.sinh(sk_l) / sqrt_k;
  }
  mat2[0][0] = cx;
  mat2[0][1] = sx / rel_p;
  mat2[1][0] = k1 * sx * rel_p;
  mat2[1][1] = cx;
  zc[0] = k1 * (-cx * sx + length) / 4;
  zc[1] = -k1 * (sx * sx) / (2 * rel_p);
  zc[2] = -(cx * sx + length) / (4 * (rel_p * rel_p));
}

// low_energy_z_correction, bmad/low_level/low_energy_z_correction.f90:22-57
double low_energy_z_correction(const Coord& orbit, const Ele& ele, double ds) {
  double mass = ele.p->mass;
  double p0c = orbit.p0c;
  double e_tot = ele.p->e_tot;
  double beta0 = p0c / e_tot;
  double pz = orbit.vec[5];
  double b0pz = beta0 * pz;
  double dz;
  if (mass * (b0pz * b0pz) < 3e-7 * e_tot) {
    double me = mass / e_tot;
    double b02 = beta0 * beta0;
    double f = b02 * (2 * b02 - (me * me) / 2);
    dz = ds * pz * (1 - 3 * (pz * b02) / 2 + (pz * pz) * f) * (me * me);
  } else {
    dz = ds * (orbit.beta - beta0) / beta0;
  }
  return dz;
}

// tilt_coords, bmad/code/tilt_coords.f90:18-53
void tilt_coords(double tilt_val, double* coord) {
  if (tilt_val == 0) return;
  double sin_ang = lm.sin(tilt_val), cos_ang = lm.cos(tilt_val);
  double x = coord[0], y = coord[2];
  coord[0] = cos_ang * x + sin_ang * y;
  coord[2] = -sin_ang * x + cos_ang * y;
  double px = coord[1], py = coord[3];
  coord[1] = cos_ang * px + sin_ang * py;
  coord[3] = -sin_ang * px + cos_ang * py;
}

// floor_angles_to_w_mat, bmad/geometry/floor_angles_to_w_mat.f90
void floor_angles_to_w_mat(double theta, double phi, double psi, double w[3][3], bool inverse) {
  double s_the = lm.sin(theta), c_the = lm.cos(theta);
  double s_phi = lm.sin(phi), c_phi = lm.cos(phi);
  double s_psi = lm.sin(psi), c_psi = lm.cos(psi);
  if (!inverse) {
    w[0][0] = c_the * c_psi - s_the * s_phi * s_psi;
    w[0][1] = -c_the * s_psi - s_the * s_phi * c_psi;
    w[0][2] = s_the * c_phi;
    w[1][0] = c_phi * s_psi;
    w[1][1] = c_phi * c_psi;
    w[1][2] = s_phi;
    w[2][0] = -s_the * c_psi - c_the * s_phi * s_psi;
    w[2][1] = s_the * s_psi - c_the * s_phi * c_psi;
    w[2][2] = c_the * c_phi;
  } else {
    w[0][0] = c_the * c_psi - s_the * s_phi * s_psi;
    w[0][1] = c_phi * s_psi;
    w[0][2] = -s_the * c_psi - c_the * s_phi * s_psi;
    w[1][0] = -c_the * s_psi - s_the * s_phi * c_psi;
    w[1][1] = c_phi * c_psi;
    w[1][2] = s_the * s_psi - c_the * s_phi * c_psi;
    w[2][0] = s_the * c_phi;
    w[2][1] = s_phi;
    w[2][2] = c_the * c_phi;
  }
}

// Fortran matmul(w(3,3), r(3)) with the inlined j-order summation.
void matvec3(const double w[3][3], const double r[3], double out[3]) {
  for (int i = 0; i < 3; i++) {
    double acc = 0;
    for (int j = 0; j < 3; j++) acc = acc + w[i][j] * r[j];
    out[i] = acc;
  }
}

// ---- bend geometry for misaligned bends -----------------------------------------------------

// cos_one, sim_utils/special_functions/cos_one.f90:16-27
double cos_one(double angle) {
  double s = lm.sin(angle / 2);
  return -2 * (s * s);
}

enum { x_axis = 1, y_axis = 2, z_axis = 3 };

// rotate_vec, sim_utils/math/rotation_3d_mod.f90:737-760
void rotate_vec(double v[3], int axis, double angle) {
  if (angle == 0) return;
  double ca = lm.cos(angle), sa = lm.sin(angle);
  if (axis == x_axis) {
    double a = ca * v[1] - sa * v[2], b = sa * v[1] + ca * v[2];
    v[1] = a; v[2] = b;
  } else if (axis == y_axis) {
    double a = sa * v[2] + ca * v[0], b = ca * v[2] - sa * v[0];
    v[0] = a; v[2] = b;
  } else {
    double a = ca * v[0] - sa * v[1], b = sa * v[0] + ca * v[1];
    v[0] = a; v[1] = b;
  }
}

// rotate_mat (rotation applied from the left), rotation_3d_mod.f90:781-845
void rotate_mat(double m[3][3], int axis, double angle) {
  if (angle == 0) return;
  double ca = lm.cos(angle), sa = lm.sin(angle);
  for (int k = 0; k < 3; k++) {
    if (axis == x_axis) {
      double a = ca * m[1][k] - sa * m[2][k], b = sa * m[1][k] + ca * m[2][k];
      m[1][k] = a; m[2][k] = b;
    } else if (axis == y_axis) {
      double a = sa * m[2][k] + ca * m[0][k], b = ca * m[2][k] - sa * m[0][k];
      m[0][k] = a; m[2][k] = b;
    } else {
      double a = ca * m[0][k] - sa * m[1][k], b = sa * m[0][k] + ca * m[1][k];
      m[0][k] = a; m[1][k] = b;
    }
  }
}

// Fortran matmul of two 3x3 matrices (j-order summation).
void matmul3(const double a[3][3], const double b[3][3], double out[3][3]) {
  double t[3][3];
  for (int i = 0; i < 3; i++)
    for (int k = 0; k < 3; k++) {
      double acc = 0;
      for (int j = 0; j < 3; j++) acc = acc + a[i][j] * b[j][k];
      t[i][k] = acc;
    }
  std::memcpy(out, t, sizeof(t));
}

struct FloorPos {  // floor_position_struct (r, w)
  double r[3];
  double w[3][3];
};

void apply_w(const double ws[3][3], FloorPos& pos) {  // r = ws r, w = ws w
  double r2[3];
  matvec3(ws, pos.r, r2);
  std::memcpy(pos.r, r2, sizeof(r2));
  matmul3(ws, pos.w, pos.w);
}

// bend_shift, bmad/geometry/bend_shift.f90:19-61; has_tilt: the optional ref_tilt is present.
FloorPos bend_shift(const FloorPos& p1, double g, double delta_s, bool has_tilt = false, double ref_tilt = 0) {
  double angle = delta_s * g;
  FloorPos p2 = p1;
  if (angle == 0) {
    p2.r[2] = p2.r[2] - delta_s;
    return p2;
  }
  double tlt = has_tilt ? ref_tilt : 0.0;
  double S[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  if (tlt != 0) {
    rotate_mat(S, z_axis, -ref_tilt);
    rotate_mat(S, y_axis, angle);
    rotate_mat(S, z_axis, ref_tilt);
  } else {
    rotate_mat(S, y_axis, angle);
  }
  double L[3] = {cos_one(angle) / g, 0.0 / g, -lm.sin(angle) / g};
  if (has_tilt) rotate_vec(L, z_axis, ref_tilt);
  double r2[3];
  matvec3(S, p1.r, r2);
  for (int i = 0; i < 3; i++) p2.r[i] = r2[i] + L[i];
  matmul3(S, p1.w, p2.w);
  return p2;
}

// w_mat_for_tilt, bmad/geometry/w_mat_for_tilt.f90:14-38
void w_mat_for_tilt(double tilt, double w[3][3]) {
  double c = lm.cos(tilt), s = lm.sin(tilt);
  double m[3][3] = {{c, -s, 0.0}, {s, c, 0.0}, {0.0, 0.0, 1.0}};
  std::memcpy(w, m, sizeof(m));
}

// offset_particle, bmad/code/offset_particle.f90:66-530 (drift_to the element ends, no roll);
// set_hvkicks and set_tilt as given.
int offset_particle(const Ele& ele, int set, Coord& orbit, bool set_tilt, bool set_hvkicks) {
  const bmadgpu_element* e = ele.e;
  const bmadgpu_param* p = ele.p;
  int key = e->key;
  bool has_orient = key_has_orientation(key);
  bool set_hv = set_hvkicks && e->is_on && key_has_hkick(key);
  bool set_t = set_tilt && has_orient;
  double length = e->l;
  double L_half = 0.5 * length;
  int sign_z_vel = 1;
  double s_pos0 = set ? 0 : length;
  double ds_center = L_half - s_pos0;
  double s_target = set ? (1 - sign_z_vel) * L_half : (1 + 1) * L_half;
  bool drift_to = has_orient;  // upstream_end (set) / downstream_end (unset) when no s_pos
  double rel_p = 1 + orbit.vec[5];
  double charge_dir = 1.0 * sign_z_vel;  // rel_tracking_charge * sign_z_vel * time_dir
  bool set_hv1 = set_hv;  // quads, sbends, sextupoles, ... (not kickers / elseparators)

  double x_off = 0, y_off = 0, z_off = 0, xp = 0, yp = 0;
  bool is_misaligned = false;
  if (has_orient) {
    x_off = e->x_offset; y_off = e->y_offset; z_off = e->z_offset;
    xp = e->x_pitch; yp = e->y_pitch;
    is_misaligned = (x_off != 0 || y_off != 0 || z_off != 0 || xp != 0 || yp != 0 ||
                     (key == BMADGPU_SBEND && e->roll != 0));
  }
  const double roll = (key == BMADGPU_SBEND) ? e->roll : 0.0;
  const bool bend_geom = is_misaligned && key == BMADGPU_SBEND && (e->g != 0 || ele.ref_tilt_tot != 0 || roll != 0);
  const double g = e->g, ref_tilt = ele.ref_tilt_tot;
  // ele_misalignment_L_S_calc (bmad/geometry/ele_misalignment_L_S_calc.f90:16-50): L_mis = the
  // offsets, moved by the roll about the bend's chord; S_mis = floor_angles_to_w_mat(x_pitch,
  // y_pitch, roll). angle = l g, rho = 1/g (0 for g = 0), attribute_bookkeeper.f90:763-770.
  double L_mis[3] = {x_off, y_off, z_off};
  if (bend_geom && roll != 0) {
    const double angle = e->l * g, rho = (g == 0) ? 0.0 : 1 / g;
    double Lc[3] = {rho * cos_one(angle / 2), rho * 0.0, rho * lm.sin(angle / 2)};
    rotate_vec(Lc, y_axis, angle / 2);
    rotate_vec(Lc, z_axis, ref_tilt);
    for (int i = 0; i < 3; i++) L_mis[i] = L_mis[i] - Lc[i];
    rotate_vec(Lc, z_axis, roll);
    for (int i = 0; i < 3; i++) L_mis[i] = L_mis[i] + Lc[i];
  }

  if (set) {
    double s_body;
    if (bend_geom) {
      // offset_particle.f90:204-227, 247-257
      FloorPos pos = {{orbit.vec[0], orbit.vec[2], 0.0}, {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}};
      pos = bend_shift(pos, g, 1 * ds_center, true, ref_tilt);
      double ws[3][3], wt[3][3];
      floor_angles_to_w_mat(xp, yp, roll, ws, false);
      for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) wt[i][j] = ws[j][i];
      double d[3] = {pos.r[0] - L_mis[0], pos.r[1] - L_mis[1], pos.r[2] - L_mis[2]};
      std::memcpy(pos.r, d, sizeof(d));
      apply_w(wt, pos);
      if (ref_tilt != 0) {
        pos = bend_shift(pos, g, -L_half, true, ref_tilt);
        double wtilt[3][3];
        w_mat_for_tilt(-ref_tilt, wtilt);
        apply_w(wtilt, pos);
        pos = bend_shift(pos, g, L_half);
      }
      pos = bend_shift(pos, g, -sign_z_vel * 1 * L_half);
      pos.r[2] = pos.r[2] + (1 - sign_z_vel * 1) * L_half;
      s_body = pos.r[2];
      double pz = rel_p * rel_p - orbit.vec[1] * orbit.vec[1] - orbit.vec[3] * orbit.vec[3];
      if (pz <= 0) {
        orbit.state = BMADGPU_LOST_PZ;
      } else {
        double p_vec0[3] = {orbit.vec[1], orbit.vec[3], sign_z_vel * std::sqrt(pz)}, p_vec[3];
        matvec3(pos.w, p_vec0, p_vec);
        orbit.vec[1] = p_vec[0];
        orbit.vec[3] = p_vec[1];
        orbit.vec[0] = pos.r[0];
        orbit.vec[2] = pos.r[1];
      }
    } else if (is_misaligned) {
      double r[3] = {orbit.vec[0] - x_off, orbit.vec[2] - y_off, 0.0 - (z_off + 1 * ds_center)};
      double ws[3][3], w[3][3], r2[3];
      floor_angles_to_w_mat(xp, yp, 0.0, ws, true);
      matvec3(ws, r, r2);
      for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) w[i][j] = ws[i][j];
      r2[2] = r2[2] + L_half;
      s_body = r2[2];
      double pz = rel_p * rel_p - orbit.vec[1] * orbit.vec[1] - orbit.vec[3] * orbit.vec[3];
      if (pz <= 0) {
        orbit.state = BMADGPU_LOST_PZ;
      } else {
        double p_vec0[3] = {orbit.vec[1], orbit.vec[3], sign_z_vel * std::sqrt(pz)}, p_vec[3];
        matvec3(w, p_vec0, p_vec);
        orbit.vec[1] = p_vec[0];
        orbit.vec[3] = p_vec[1];
        orbit.vec[0] = r2[0];
        orbit.vec[2] = r2[1];
      }
    } else {
      if (key == BMADGPU_SBEND && e->ref_tilt != 0) tilt_coords(e->ref_tilt, orbit.vec);
      s_body = s_pos0;
    }
    double ds = s_target - s_body;
    if (std::fabs(ds) > 1e-14 && drift_to && orbit.state == BMADGPU_ALIVE)
      track_a_drift(orbit, ds, p, false, 1);
    if (set_hv1) {
      orbit.vec[1] = orbit.vec[1] + 0.5 * charge_dir * e->hkick;
      orbit.vec[3] = orbit.vec[3] + 0.5 * charge_dir * e->vkick;
    }
    if (set_t && key != BMADGPU_SBEND && ele.tilt_tot != 0) tilt_coords(ele.tilt_tot, orbit.vec);
  } else {
    if (set_t && key != BMADGPU_SBEND) tilt_coords(-ele.tilt_tot, orbit.vec);
    if (set_hv1) {
      orbit.vec[1] = orbit.vec[1] + 0.5 * charge_dir * e->hkick;
      orbit.vec[3] = orbit.vec[3] + 0.5 * charge_dir * e->vkick;
    }
    double s_lab;
    if (bend_geom) {
      // offset_particle.f90:399-425, 445-457
      FloorPos pos = {{orbit.vec[0], orbit.vec[2], 0.0}, {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}};
      pos = bend_shift(pos, g, ds_center);
      if (ref_tilt != 0) {
        pos = bend_shift(pos, g, -L_half);
        double wtilt[3][3];
        w_mat_for_tilt(ref_tilt, wtilt);
        apply_w(wtilt, pos);
        pos = bend_shift(pos, g, L_half, true, ref_tilt);
      }
      double ws[3][3];
      floor_angles_to_w_mat(xp, yp, roll, ws, false);
      apply_w(ws, pos);
      for (int i = 0; i < 3; i++) pos.r[i] = pos.r[i] + L_mis[i];
      pos = bend_shift(pos, g, sign_z_vel * 1 * L_half, true, ref_tilt);
      pos.r[2] = pos.r[2] + (1 + sign_z_vel * 1) * L_half;
      s_lab = pos.r[2];
      double pz = rel_p * rel_p - orbit.vec[1] * orbit.vec[1] - orbit.vec[3] * orbit.vec[3];
      if (pz <= 0) {
        orbit.state = BMADGPU_LOST_PZ;
      } else {
        double p_vec0[3] = {orbit.vec[1], orbit.vec[3], sign_z_vel * std::sqrt(pz)}, p_vec[3];
        matvec3(pos.w, p_vec0, p_vec);
        orbit.vec[1] = p_vec[0];
        orbit.vec[3] = p_vec[1];
        orbit.vec[0] = pos.r[0];
        orbit.vec[2] = pos.r[1];
      }
    } else if (is_misaligned) {
      double r[3] = {orbit.vec[0], orbit.vec[2], 0.0};
      r[2] = r[2] - ds_center;
      double ws[3][3], r2[3];
      floor_angles_to_w_mat(xp, yp, 0.0, ws, false);
      matvec3(ws, r, r2);
      r2[0] = r2[0] + x_off;
      r2[1] = r2[1] + y_off;
      r2[2] = r2[2] + (z_off + L_half);
      s_lab = r2[2];
      double pz = rel_p * rel_p - orbit.vec[1] * orbit.vec[1] - orbit.vec[3] * orbit.vec[3];
      if (pz <= 0) {
        orbit.state = BMADGPU_LOST_PZ;
      } else {
        double p_vec0[3] = {orbit.vec[1], orbit.vec[3], sign_z_vel * std::sqrt(pz)}, p_vec[3];
        matvec3(ws, p_vec0, p_vec);
        orbit.vec[1] = p_vec[0];
        orbit.vec[3] = p_vec[1];
        orbit.vec[0] = r2[0];
        orbit.vec[2] = r2[1];
      }
    } else {
      if (key == BMADGPU_SBEND && e->ref_tilt != 0) tilt_coords(-e->ref_tilt, orbit.vec);
      s_lab = s_pos0;
    }
    double ds = s_target - s_lab;
    if (std::fabs(ds) > 1e-14 && drift_to && orbit.state == BMADGPU_ALIVE)
      track_a_drift(orbit, ds, p, false, 1);
  }
  return 0;
}

// ---------------------------------------------------------------------------------------------
// Aperture and orbit checks

// orbit_too_large, bmad/low_level/orbit_too_large.f90:26-120
bool orbit_too_large(Coord& orbit, const bmadgpu_param* p) {
  double lim = p->max_aperture_limit;
  if (orbit.vec[0] > lim) { orbit.state = BMADGPU_LOST_POS_X; return true; }
  if (-orbit.vec[0] > lim) { orbit.state = BMADGPU_LOST_NEG_X; return true; }
  if (orbit.vec[2] > lim) { orbit.state = BMADGPU_LOST_POS_Y; return true; }
  if (-orbit.vec[2] > lim) { orbit.state = BMADGPU_LOST_NEG_Y; return true; }
  double rel_p = 1 + orbit.vec[5];
  if (rel_p < 0) { orbit.state = BMADGPU_LOST_PZ; return true; }
  double f_unstable = orbit.vec[1] * orbit.vec[1] + orbit.vec[3] * orbit.vec[3] - rel_p * rel_p;
  if (f_unstable > 0) {
    if (std::fabs(orbit.vec[1]) > std::fabs(orbit.vec[3])) {
      orbit.state = (orbit.vec[1] > 0) ? BMADGPU_LOST_POS_X : BMADGPU_LOST_NEG_X;
    } else {
      orbit.state = (orbit.vec[3] > 0) ? BMADGPU_LOST_POS_Y : BMADGPU_LOST_NEG_Y;
    }
    return true;
  }
  return false;
}

// at_this_ele_end, bmad/code/at_this_ele_end.f90:16-61 (now_at = entrance_end or exit_end)
bool at_this_ele_end(int now_at, int where_at) {
  if (where_at == BMADGPU_NO_END) return false;
  if (where_at == BMADGPU_CONTINUOUS || where_at == 7) return true;
  if (now_at == BMADGPU_ENTRANCE_END) return where_at == BMADGPU_ENTRANCE_END || where_at == BMADGPU_BOTH_ENDS;
  if (now_at == BMADGPU_EXIT_END) return where_at == BMADGPU_EXIT_END || where_at == BMADGPU_BOTH_ENDS;
  return false;
}

// check_this_limit (check_aperture_limit.f90:344-356): a phase-space window centre +- width2
void check_this_limit(Coord& orb, double coord, double width2, double center, double* unstable_factor) {
  if (width2 == 0) return;
  if (coord > center - width2 && coord < center + width2) return;
  orb.state = BMADGPU_LOST;
  *unstable_factor = std::max((center - width2) - coord, coord - (center + width2));
}

// elliptical_params_setup (check_aperture_limit.f90:361-387); false on limits set on one side only
bool elliptical_params_setup(double lim1, double lim2, double* pos, double* width2, double* center,
                             const bmadgpu_param* p) {
  if ((lim1 == 0 && lim2 != 0) || (lim1 != 0 && lim2 == 0)) return false;
  *width2 = (lim2 - lim1) / 2;
  *center = (lim2 + lim1) / 2;
  *pos = *pos - *center;
  if (*width2 == 0) *width2 = p->max_aperture_limit;
  *width2 = std::max(*width2, 0.0);
  return true;
}

// check_aperture_limit, bmad/low_level/check_aperture_limit.f90:30-387 (rectangular and
// elliptical apertures with the collimators' phase-space windows, offset_moves_aperture = F, no
// wall_transition). unstable: param%unstable_factor on return (may be null).
int check_aperture_limit(Coord& orb, const Ele& ele, int particle_at, double* unstable = nullptr) {
  const bmadgpu_element* e = ele.e;
  double unstable_factor = 0;
  if (unstable) *unstable = 0;
  if (orbit_too_large(orb, ele.p)) return 0;
  if (!ele.p->aperture_limit_on) return 0;
  int physical_end = (particle_at == first_track_edge) ? BMADGPU_ENTRANCE_END : BMADGPU_EXIT_END;
  if (!at_this_ele_end(physical_end, e->aperture_at)) return 0;
  // momentum and longitudinal windows, :113-151
  if (e->key == BMADGPU_ECOLLIMATOR) {
    const double pairs[2][4] = {{e->px_aperture_width2, e->py_aperture_width2, e->px_aperture_center,
                                 e->py_aperture_center},
                                {e->z_aperture_width2, e->pz_aperture_width2, e->z_aperture_center,
                                 e->pz_aperture_center}};
    for (int k = 0; k < 2; k++) {
      const double xw = pairs[k][0], yw = pairs[k][1], x0 = pairs[k][2], y0 = pairs[k][3];
      const double u = orb.vec[k == 0 ? 1 : 4], v = orb.vec[k == 0 ? 3 : 5];
      if (xw == 0 || yw == 0) {
        check_this_limit(orb, u, xw, x0, &unstable_factor);
        check_this_limit(orb, v, yw, y0, &unstable_factor);
      } else {
        const double r = ((u - x0) / xw) * ((u - x0) / xw) + ((v - y0) / yw) * ((v - y0) / yw);
        if (r > 1) {
          orb.state = BMADGPU_LOST;
          unstable_factor = std::sqrt(r) - 1;
        }
      }
    }
  } else if (e->key == BMADGPU_RCOLLIMATOR) {
    check_this_limit(orb, orb.vec[1], e->px_aperture_width2, e->px_aperture_center, &unstable_factor);
    check_this_limit(orb, orb.vec[3], e->py_aperture_width2, e->py_aperture_center, &unstable_factor);
    check_this_limit(orb, orb.vec[4], e->z_aperture_width2, e->z_aperture_center, &unstable_factor);
    check_this_limit(orb, orb.vec[5], e->pz_aperture_width2, e->pz_aperture_center, &unstable_factor);
  }
  double x_particle = orb.vec[0], y_particle = orb.vec[2];
  double x1_lim = -e->x1_limit, x2_lim = e->x2_limit, y1_lim = -e->y1_limit, y2_lim = e->y2_limit;
  if (e->aperture_type == BMADGPU_APERTURE_RECTANGULAR || e->aperture_type == BMADGPU_APERTURE_AUTO) {
    if (x1_lim != 0 && x_particle < x1_lim) {
      double f = std::fabs((x_particle - x1_lim) / (x2_lim - x1_lim));
      if (f > unstable_factor) { orb.state = BMADGPU_LOST_NEG_X; unstable_factor = f; }
    }
    if (x2_lim != 0 && x_particle > x2_lim) {
      double f = std::fabs((x_particle - x2_lim) / (x2_lim - x1_lim));
      if (f > unstable_factor) { orb.state = BMADGPU_LOST_POS_X; unstable_factor = f; }
    }
    if (y1_lim != 0 && y_particle < y1_lim) {
      double f = std::fabs((y_particle - y1_lim) / (y2_lim - y1_lim));
      if (f > unstable_factor) { orb.state = BMADGPU_LOST_NEG_Y; unstable_factor = f; }
    }
    if (y2_lim != 0 && y_particle > y2_lim) {
      double f = std::fabs((y_particle - y2_lim) / (y2_lim - y1_lim));
      if (f > unstable_factor) { orb.state = BMADGPU_LOST_POS_Y; unstable_factor = f; }
    }
    if (unstable) *unstable = unstable_factor;
    return 0;
  }
  if (e->aperture_type == BMADGPU_APERTURE_ELLIPTICAL) {
    double x_width2, x0, y_width2, y0;
    if (!elliptical_params_setup(x1_lim, x2_lim, &x_particle, &x_width2, &x0, ele.p)) return 0;
    if (!elliptical_params_setup(y1_lim, y2_lim, &y_particle, &y_width2, &y0, ele.p)) return 0;
    const double rx = x_particle / x_width2, ry = y_particle / y_width2;
    const double r = rx * rx + ry * ry;
    if (r < 1) {
      if (unstable) *unstable = unstable_factor;
      return 0;
    }
    if (std::fabs(x_particle / x_width2) > std::fabs(y_particle / y_width2)) {
      orb.state = (x_particle > 0) ? BMADGPU_LOST_POS_X : BMADGPU_LOST_NEG_X;
    } else {
      orb.state = (y_particle > 0) ? BMADGPU_LOST_POS_Y : BMADGPU_LOST_NEG_Y;
    }
    unstable_factor = std::sqrt(r) - 1;
    if (unstable) *unstable = unstable_factor;
    return 0;
  }
  return BMADGPU_EUNSUPPORTED;
}

// ---------------------------------------------------------------------------------------------
// Edge kicks

// hwang_bend_edge_kick, bmad/modules/fringe_mod.f90:241-419 (time_dir = +1); mat6 optional.
void hwang_bend_edge_kick(const Ele& ele, int particle_at, Coord& orb, double* mat6) {
  const bmadgpu_element* e = ele.e;
  double c_dir = 1.0;
  int element_end = (particle_at == first_track_edge) ? BMADGPU_ENTRANCE_END : BMADGPU_EXIT_END;
  int fringe_type = e->fringe_type;
  double e_factor = 1 / (1 + orb.vec[5]);
  double td = 1.0;
  double g_tot, k1;
  if (e->is_on) {
    g_tot = (e->g + e->dg) * c_dir;
    k1 = e->k1;
  } else {
    g_tot = 0;
    k1 = 0;
  }
  double ee, fint_gap;
  if (element_end == BMADGPU_ENTRANCE_END) {
    ee = e->e1;
    fint_gap = e->fint * e->hgap;
  } else {
    ee = e->e2;
    fint_gap = e->fintx * e->hgapx;
  }
  if (fringe_type == BMADGPU_FRINGE_HARD_EDGE_ONLY || fringe_type == BMADGPU_FRINGE_SAD_FULL) fint_gap = 0;
  double cos_e = lm.cos(ee), sin_e = lm.sin(ee);
  double tan_e = sin_e / cos_e, sec_e = 1 / cos_e;
  double gt = g_tot * tan_e;
  double gt2 = g_tot * (tan_e * tan_e);
  double gs2 = g_tot * (sec_e * sec_e);
  double k1_tane = k1 * tan_e * c_dir;
  double fg_factor = 2 * fint_gap * gs2 * g_tot * sec_e * (1 + sin_e * sin_e);
  double v[6];
  for (int i = 0; i < 6; i++) v[i] = orb.vec[i];
  double dx, dpx, dy, dpy, dz;
  double km[6][6];
  for (int i = 0; i < 6; i++) for (int j = 0; j < 6; j++) km[i][j] = (i == j) ? 1 : 0;
  double v1 = v[0], v2 = v[1], v3 = v[2], v4 = v[3];
  if (particle_at == first_track_edge) {  // entering_element
    dx = (-gt2 * (v1 * v1) + gs2 * (v3 * v3)) * e_factor / 2;
    dpx = (gt * g_tot * (1 + 2 * (tan_e * tan_e)) * (v3 * v3) / 2 + gt2 * (v1 * v2 - v3 * v4) +
           k1_tane * ((v1 * v1) - (v3 * v3))) * e_factor;
    dy = gt2 * v1 * v3 * e_factor;
    dpy = (fg_factor * v3 - gt2 * v1 * v4 - (g_tot + gt2) * v2 * v3 - 2 * k1_tane * v1 * v3) * e_factor;
    dz = (e_factor * e_factor) * 0.5 *
         ((v3 * v3) * fg_factor + (v1 * v1 * v1) * (4.0 * k1_tane - gt * gt2) / 6.0 +
          0.5 * v1 * (v3 * v3) * (-4.0 * k1_tane + gt * gs2) +
          ((v1 * v1) * v2 - 2.0 * v1 * v3 * v4) * gt2 - v2 * (v3 * v3) * gs2);
    orb.vec[0] = v[0] + td * dx;
    orb.vec[1] = v[1] + td * (dpx + gt * v[0]);
    orb.vec[2] = v[2] + td * dy;
    orb.vec[3] = v[3] + td * (dpy - gt * v[2]);
    orb.vec[4] = v[4] + td * dz;
    if (mat6) {
      km[0][0] = 1 - gt2 * v1 * e_factor;
      km[0][2] = gs2 * v3 * e_factor;
      km[1][0] = gt + (gt2 * v2 + 2 * k1_tane * v1) * e_factor;
      km[1][1] = 1 + (gt2 * v1) * e_factor;
      km[1][2] = (-gt2 * v4 - 2 * k1_tane * v3 + gt * g_tot * (1 + 2 * (tan_e * tan_e)) * v3) * e_factor;
      km[1][3] = (-gt2 * v3) * e_factor;
      km[2][0] = gt2 * v3 * e_factor;
      km[2][2] = 1 + gt2 * v1 * e_factor;
      km[3][0] = (-gt2 * v4 - 2 * k1_tane * v3) * e_factor;
      km[3][1] = -(g_tot + gt2) * v3 * e_factor;
      km[3][2] = -gt + (fg_factor - (g_tot + gt2) * v2 - 2 * k1_tane * v1) * e_factor;
      km[3][3] = 1 - gt2 * v1 * e_factor;
      km[4][5] = (fg_factor * (v3 * v3) / 2 + (4 * k1_tane - gt * gt2) * (v1 * v1 * v1) / 12 +
                  (-4 * k1_tane + gt * gs2) * v1 * (v3 * v3) / 4 +
                  gt2 * ((v1 * v1) * v2 - 2 * v1 * v3 * v4) / 2 - (g_tot + gt2) * v2 * (v3 * v3) / 2) *
                 (e_factor * e_factor);
    }
  } else {
    dx = (gt2 * (v1 * v1) - gs2 * (v3 * v3)) * e_factor / 2;
    dpx = (gt2 * (v3 * v4 - v1 * v2) + k1_tane * ((v1 * v1) - (v3 * v3)) - gt * gt2 * ((v1 * v1) + (v3 * v3)) / 2) *
          e_factor;
    dy = -gt2 * v1 * v3 * e_factor;
    dpy = (fg_factor * v3 + gt2 * v1 * v4 + (g_tot + gt2) * v2 * v3 + (gt * gs2 - 2 * k1_tane) * v1 * v3) * e_factor;
    dz = (e_factor * e_factor) * 0.5 *
         ((v3 * v3) * fg_factor + (v1 * v1 * v1) * (4.0 * k1_tane - gt * gt2) / 6.0 +
          0.5 * v1 * (v3 * v3) * (-4.0 * k1_tane + gt * gs2) -
          ((v1 * v1) * v2 - 2.0 * v1 * v3 * v4) * gt2 + v2 * (v3 * v3) * gs2);
    orb.vec[0] = v[0] + td * dx;
    orb.vec[1] = v[1] + td * (dpx + gt * v[0]);
    orb.vec[2] = v[2] + td * dy;
    orb.vec[3] = v[3] + td * (dpy - gt * v[2]);
    orb.vec[4] = v[4] + td * dz;
    if (mat6) {
      km[0][0] = 1 + gt2 * v1 * e_factor;
      km[0][2] = -gs2 * v3 * e_factor;
      km[1][0] = gt + (-gt2 * v2 + 2 * k1_tane * v1 - gt * gt2 * v1) * e_factor;
      km[1][1] = 1 - gt2 * v1 * e_factor;
      km[1][2] = (gt2 * v4 - 2 * k1_tane * v3 - gt * gt2 * v3) * e_factor;
      km[1][3] = gt2 * v3 * e_factor;
      km[2][0] = -gt2 * v3 * e_factor;
      km[2][2] = 1 - gt2 * v1 * e_factor;
      km[3][0] = (gt2 * v4 + (gt * gs2 - 2 * k1_tane) * v3) * e_factor;
      km[3][1] = (g_tot + gt2) * v3 * e_factor;
      km[3][2] = -gt + (fg_factor + (g_tot + gt2) * v2 + (gt * gs2 - 2 * k1_tane) * v1) * e_factor;
      km[3][3] = 1 + gt2 * v1 * e_factor;
      km[4][5] = (fg_factor * (v3 * v3) / 2 + (4 * k1_tane - gt * gt2) * (v1 * v1 * v1) / 12 +
                  (-4 * k1_tane + gt * gs2) * v1 * (v3 * v3) / 4 +
                  gt2 * (-(v1 * v1) * v2 + 2 * v1 * v3 * v4) / 2 + (g_tot + gt2) * v2 * (v3 * v3) / 2) *
                 (e_factor * e_factor);
    }
  }
  if (mat6) {
    km[0][5] = -dx * e_factor;
    km[1][5] = -dpx * e_factor;
    km[2][5] = -dy * e_factor;
    km[3][5] = -dpy * e_factor;
    for (int j = 0; j < 4; j++)
      km[4][j] = -km[1][5] * km[0][j] + km[0][5] * km[1][j] - km[3][5] * km[2][j] + km[2][5] * km[3][j];
    double out[6][6];
    for (int i = 0; i < 6; i++)
      for (int j = 0; j < 6; j++) {
        double acc = 0;
        for (int k = 0; k < 6; k++) acc = acc + km[i][k] * mat6[k * 6 + j];
        out[i][j] = acc;
      }
    for (int i = 0; i < 6; i++) for (int j = 0; j < 6; j++) mat6[i * 6 + j] = out[i][j];
  }
}

// apply_energy_kick, bmad/low_level/apply_energy_kick.f90:23-74
void apply_energy_kick(double dE, Coord& orbit, const bmadgpu_param* p) {
  double mc2 = p->mass;
  double p0c = orbit.p0c;
  double pc = (1 + orbit.vec[5]) * p0c;
  double beta_old = orbit.beta;
  double E_old = pc / orbit.beta;
  double E_new = E_old + dE;
  if (E_new < mc2) {
    orbit.vec[5] = -1;
    orbit.beta = 0;
    orbit.state = BMADGPU_LOST_PZ;
    return;
  }
  orbit.vec[5] = orbit.vec[5] + (1 + orbit.vec[5]) * sqrt_one((2 * E_old * dE + dE * dE) / (pc * pc));
  double pc_new = p0c * (1 + orbit.vec[5]);
  double beta_new = pc_new / E_new;
  orbit.vec[4] = orbit.vec[4] * beta_new / beta_old;
  orbit.beta = beta_new;
}

// electric_longitudinal_fringe, bmad/low_level/apply_element_edge_kick.f90:283-329
// (bmad_standard field_calc, non-exact multipoles)
void electric_longitudinal_fringe(Coord& orb, const Ele& ele, const double* a_pole_elec,
                                  const double* b_pole_elec, int ix_elec_max, double at_sign) {
  if (ele.e->l == 0) return;
  if (ix_elec_max <= -1) return;
  double ff = at_sign * ele.p->charge;
  double xr = 1, xi = 0;            // xiy
  double cr = orb.vec[0], ci = orb.vec[2];  // c_vec
  double phi = 0, E_r0 = 0, E_r1 = 0;
  for (int i = 0; i <= ix_elec_max; i++) {
    double xor_ = xr, xoi = xi;
    double nr = xr * cr - xi * ci, ni = xr * ci + xi * cr;
    xr = nr; xi = ni;
    if (a_pole_elec[i] == 0 && b_pole_elec[i] == 0) continue;
    double ar = b_pole_elec[i], ai = -a_pole_elec[i];  // ab_elec
    double re_cur = ar * xr - ai * xi;
    phi = phi - re_cur / (i + 1);
    double re_old = ar * xor_ - ai * xoi, im_old = ar * xoi + ai * xor_;
    E_r0 = E_r0 + re_old;
    E_r1 = E_r1 + (-im_old);
  }
  apply_energy_kick(-ff * phi, orb, ele.p);
  (void)E_r0; (void)E_r1;  // only enter the transfer matrix
}

// fringe_here, bmad/code/fringe_here.f90:15-35
bool fringe_here(const Ele& ele, int particle_at) {
  int physical_end = (particle_at == first_track_edge) ? BMADGPU_ENTRANCE_END : BMADGPU_EXIT_END;
  if (ele.e->fringe_type == BMADGPU_FRINGE_NONE) return false;
  return at_this_ele_end(physical_end, ele.e->fringe_at);
}

// Complex numbers with gfortran's operations (products written out, no special-value rules).
struct Cx {
  double re, im;
};
Cx cmul(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
Cx cadd(Cx a, Cx b) { return {a.re + b.re, a.im + b.im}; }
Cx cscale(double f, Cx a) { return {f * a.re, f * a.im}; }

// hard_multipole_edge_kick, bmad/modules/fringe_mod.f90:692-865 (no matrix): the hard-edge
// fringe of the quadrupole (n = 1) or sextupole (n = 2) component of a quadrupole, sbend or
// sextupole with fringe_type full (or hard_edge_only, not for sbends).
void hard_multipole_edge_kick(const Ele& ele, int particle_at, Coord& orbit) {
  const bmadgpu_element* e = ele.e;
  switch (e->fringe_type) {
    case BMADGPU_FRINGE_HARD_EDGE_ONLY:
      if (e->key == BMADGPU_SBEND) return;
      break;
    case BMADGPU_FRINGE_FULL:
      break;
    default:
      return;
  }
  if (!fringe_here(ele, particle_at)) return;
  const double charge_dir = 1.0 * 1.0 * 1.0;  // orientation * direction * rel_tracking_charge
  int n_max;
  switch (e->key) {
    case BMADGPU_QUADRUPOLE: case BMADGPU_SBEND: n_max = 1; break;
    case BMADGPU_SEXTUPOLE: n_max = 2; break;
    default: return;
  }
  const double x = orbit.vec[0], y = orbit.vec[2];
  const Cx xy = {x, y};
  Cx poly_n1 = {1, 0}, poly = xy;
  const double rel_p = 1 + orbit.vec[5];
  double fx = 0, dfx_dx = 0, dfx_dy = 0, fy = 0, dfy_dx = 0, dfy_dy = 0;
  for (int n = 1; n <= n_max; n++) {
    poly_n1 = poly;
    poly = cmul(poly, xy);
    double ap, bp;
    if (e->key == BMADGPU_SEXTUPOLE) {
      ap = 0;
      bp = e->k2;
      if (n != 2) continue;
    } else {
      ap = 0;
      bp = e->k1;
    }
    const Cx dpoly_dx = cscale(n + 1, poly_n1);
    const Cx dpoly_dy = {-dpoly_dx.im, dpoly_dx.re};  // i_imag * dpoly_dx
    const double div = 4 * (n + 2) * rel_p;
    Cx cab = cscale(charge_dir, Cx{bp, ap});
    cab = {cab.re / div, cab.im / div};
    if (particle_at == first_track_edge) cab = {-cab.re, -cab.im};
    const double cn = (double)(n + 3) / (n + 1);
    Cx xny = {x, -cn * y};
    const Cx dxny_dy = {0.0, -cn};
    fx = fx + cmul(cmul(cab, poly), xny).re;
    dfx_dx = dfx_dx + cmul(cab, cadd(cmul(dpoly_dx, xny), poly)).re;
    dfx_dy = dfx_dy + cmul(cab, cadd(cmul(dpoly_dy, xny), cmul(poly, dxny_dy))).re;
    xny = {y, cn * x};
    const Cx dxny_dx = {0.0, cn};
    fy = fy + cmul(cmul(cab, poly), xny).re;
    dfy_dx = dfy_dx + cmul(cab, cadd(cmul(dpoly_dx, xny), cmul(poly, dxny_dx))).re;
    dfy_dy = dfy_dy + cmul(cab, cadd(cmul(dpoly_dy, xny), poly)).re;
  }
  const double px = orbit.vec[1], py = orbit.vec[3];
  const double denom = (1 - dfx_dx) * (1 - dfy_dy) - dfx_dy * dfy_dx;
  orbit.vec[0] = orbit.vec[0] - fx;
  orbit.vec[1] = px + ((1.0 - dfy_dy - denom) * px + dfy_dx * py) / denom;
  orbit.vec[2] = orbit.vec[2] - fy;
  orbit.vec[3] = py + (dfx_dy * px + (1.0 - dfx_dx - denom) * py) / denom;
  orbit.vec[4] = orbit.vec[4] + (orbit.vec[1] * fx + orbit.vec[3] * fy) / rel_p;
}

// soft_quadrupole_edge_kick, bmad/modules/fringe_mod.f90:556-661 (no matrix; quadrupoles, tilt1 = 0)
void soft_quadrupole_edge_kick(const Ele& ele, int particle_at, Coord& orbit) {
  const bmadgpu_element* e = ele.e;
  if (e->fringe_type != BMADGPU_FRINGE_SOFT_EDGE_ONLY && e->fringe_type != BMADGPU_FRINGE_FULL) return;
  if (!fringe_here(ele, particle_at)) return;
  if (e->key != BMADGPU_QUADRUPOLE) return;
  const double charge_dir = 1.0 * 1.0 * 1.0;
  const double rel_p = 1 + orbit.vec[5];
  const double k1_rel = charge_dir * e->k1 / rel_p;
  double f1 = k1_rel * e->fq1;
  const double f2 = k1_rel * e->fq2;
  if (f1 == 0 && f2 == 0) return;
  if (particle_at == second_track_edge) f1 = -f1;
  const double ef1 = lm.exp(f1);
  tilt_coords(0.0, orbit.vec);
  const double v0 = orbit.vec[0], v1 = orbit.vec[1], v2 = orbit.vec[2], v3 = orbit.vec[3];
  const double vx = v1 / rel_p, vy = v3 / rel_p;
  orbit.vec[4] = orbit.vec[4] - (f1 * v0 + f2 * (1 + f1 / 2) * vx / ef1) * vx +
                 (f1 * v2 + f2 * (1 - f1 / 2) * vy * ef1) * vy;
  orbit.vec[0] = v0 * ef1 + vx * f2;
  orbit.vec[1] = v1 / ef1;
  orbit.vec[2] = v2 / ef1 - vy * f2;
  orbit.vec[3] = v3 * ef1;
  tilt_coords(-0.0, orbit.vec);
}

// bmad_rot_xz, fringe_mod.f90:1691-1771 (no matrix). Returns false on a lost particle.
bool bmad_rot_xz(double a, double vec[6]) {
  const double x = vec[0], px = vec[1], py = vec[3], delta = vec[5];
  const double pp = 1 + delta;
  double ps = pp * pp - px * px - py * py;
  if (ps <= 0) return false;
  ps = std::sqrt(ps);
  const double ca = lm.cos(a), sa = lm.sin(a);
  const double den = ps * ca - px * sa;
  const double L = x * sa / den;
  vec[0] = x * ps / den;
  vec[1] = px * ca + ps * sa;
  vec[2] = vec[2] + py * L;
  vec[4] = vec[4] - pp * L;
  return true;
}

// bmad_wedger, fringe_mod.f90:1563-1690 (no matrix): a wedge of angle a in a field g_tot.
bool bmad_wedger(double a, double g_tot, double vec[6]) {
  const double b1 = g_tot;
  if (b1 == 0) return bmad_rot_xz(a, vec);
  const double x = vec[0], px = vec[1], py = vec[3], delta = vec[5];
  const double pp = 1 + delta;
  double ps = pp * pp - px * px - py * py;
  if (ps <= 0) return false;
  ps = std::sqrt(ps);
  double pt = pp * pp - py * py;
  if (pt < 1e-10) return false;
  pt = std::sqrt(pt);
  const double ca = lm.cos(a), sa = lm.sin(a), s2a = lm.sin(2.0 * a), s2 = sa * sa;
  const double pxn = px * ca + (ps - b1 * x) * sa;
  double psn = pt * pt - pxn * pxn;
  if (psn < 1e-10) return false;
  psn = std::sqrt(psn);
  const double den = psn + ps * ca - px * sa;
  const double num = x * px * s2a + s2 * (2 * x * ps - b1 * (x * x));
  const double L = (a + lm.asin(px / pt) - lm.asin(pxn / pt)) / b1;
  vec[0] = x * ca + num / den;
  vec[1] = pxn;
  vec[2] = vec[2] + py * L;
  vec[4] = vec[4] - pp * L;
  return true;
}

// bmad_fringe_dipoler, fringe_mod.f90:1772-1933 (no matrix): the hard-edge dipole fringe with
// the fringe integral fint * hgap.
bool bmad_fringe_dipoler(double vec[6], double g_tot, double beta0, double fint, double hgap, int particle_at) {
  const double b = (particle_at == second_track_edge) ? -g_tot : g_tot;
  const double x = vec[0], px = vec[1], y = vec[2], py = vec[3], z = vec[4], delta = vec[5];
  const double pp = 1 + delta;
  double ps = pp * pp - px * px - py * py;
  if (ps <= 0) return false;
  ps = std::sqrt(ps);
  const double ee = std::sqrt(pp * pp + 1 / (beta0 * beta0) - 1);
  const double beta = pp / ee;
  const double xp = px / ps, yp = py / ps;
  const double kap = b * fint * hgap;
  const double fac2 = 1 + yp * yp;
  const double d11 = (1 + xp * xp) / ps, d21 = xp * yp / ps, d31 = -xp;
  const double d12 = xp * yp / ps, d22 = fac2 / ps, d32 = -yp;
  const double d13 = -(ee * xp / (ps * ps)), d23 = -(ee * yp / (ps * ps)), d33 = ee / ps;
  const double xf = xp / fac2;
  const double fi0 = lm.atan2(xf, 1.0) - 2 * kap * (1 + xp * xp * (2 + yp * yp)) * ps;  // atan(xp/fac2)
  const double cf = lm.cos(fi0);
  const double co2 = b / (cf * cf);
  const double co1 = co2 / (1 + xf * xf);
  const double fi1 = co1 / fac2 - 4 * kap * co2 * xp * (2 + yp * yp) * ps;
  const double fi2 = -(2 * co1 * xp * yp / (fac2 * fac2)) - 4 * kap * co2 * (xp * xp) * yp * ps;
  const double fi3 = -(2 * kap * co2 * (1 + xp * xp * (2 + yp * yp)));
  const double fi0t = b * lm.tan(fi0);
  const double bb2 = fi1 * d12 + fi2 * d22 + fi3 * d32;
  double sq = 1 - 2 * bb2 * y;
  if (sq < 0) return false;
  sq = std::sqrt(sq);
  const double ynew = 2 * y / (1 + sq);
  const double bb1 = fi1 * d11 + fi2 * d21 + fi3 * d31;
  const double bb3 = fi1 * d13 + fi2 * d23 + fi3 * d33;
  vec[0] = x + 0.5 * bb1 * (ynew * ynew);
  vec[2] = ynew;
  vec[3] = py - fi0t * ynew;
  vec[4] = z + 0.5 * beta * bb3 * (ynew * ynew);
  return true;
}

// exact_bend_edge_kick, fringe_mod.f90:1474-1562 (no matrix; the time coordinate follows from
// the element's end orbit): wedge, hard-edge dipole fringe, wedge.
void exact_bend_edge_kick(const Ele& ele, int particle_at, Coord& orb) {
  const bmadgpu_element* e = ele.e;
  const bmadgpu_param* p = ele.p;
  const double beta0 = p->p0c / p->e_tot;
  const double g_tot = e->is_on ? e->g + e->dg : 0.0;
  double edge_angle, fint, hgap;
  if (particle_at == first_track_edge) {
    edge_angle = 1 * e->e1;
    fint = e->fint;
    hgap = e->hgap;
  } else {
    edge_angle = 1 * e->e2;
    fint = e->fintx;
    hgap = e->hgapx;
  }
  double vec[6];
  for (int i = 0; i < 6; i++) vec[i] = orb.vec[i];
  bool ok;
  if (particle_at == first_track_edge) {
    ok = bmad_wedger(edge_angle, 0.0, vec) && bmad_fringe_dipoler(vec, g_tot, beta0, 1 * fint, hgap, particle_at) &&
         bmad_wedger(-edge_angle, g_tot, vec);
  } else {
    ok = bmad_wedger(-edge_angle, g_tot, vec) && bmad_fringe_dipoler(vec, g_tot, beta0, 1 * fint, hgap, particle_at) &&
         bmad_wedger(edge_angle, 0.0, vec);
  }
  if (!ok) {
    orb.state = BMADGPU_LOST_PZ;
    return;
  }
  for (int i = 0; i < 6; i++) orb.vec[i] = vec[i];
}

// apply_element_edge_kick, bmad/low_level/apply_element_edge_kick.f90:37-282, for the
// element types on the path with bmad_standard field_calc.
int apply_element_edge_kick(Coord& orb, const Ele& ele, int particle_at) {
  const bmadgpu_element* e = ele.e;
  int physical_end = (particle_at == first_track_edge) ? BMADGPU_ENTRANCE_END : BMADGPU_EXIT_END;
  if (!at_this_ele_end(physical_end, e->fringe_at)) return 0;
  double at_sign = (particle_at == first_track_edge) ? 1.0 : -1.0;
  if (orb.beta == 0) orb.state = BMADGPU_LOST;
  double a_el[n_pole_maxx + 1], b_el[n_pole_maxx + 1];
  int ix_elec_max;
  int err = multipole_ele_to_ab(ele, false, &ix_elec_max, a_el, b_el, electric, false, nullptr);
  if (err) return err;
  if (particle_at == second_track_edge) electric_longitudinal_fringe(orb, ele, a_el, b_el, ix_elec_max, at_sign);
  switch (e->key) {
    case BMADGPU_QUADRUPOLE:  // apply_element_edge_kick.f90:171-179
      if (particle_at == first_track_edge) {
        hard_multipole_edge_kick(ele, particle_at, orb);
        soft_quadrupole_edge_kick(ele, particle_at, orb);
      } else {
        soft_quadrupole_edge_kick(ele, particle_at, orb);
        hard_multipole_edge_kick(ele, particle_at, orb);
      }
      break;
    case BMADGPU_SEXTUPOLE:
      hard_multipole_edge_kick(ele, particle_at, orb);
      break;
    case BMADGPU_ELSEPARATOR:  // longitudinal fringe of the separator's field, :263-272
      if (e->l != 0) {
        const double ff = at_sign * ele.p->charge * (ele.p->p0c / e->l);
        const double phi = ff * (e->hkick * orb.vec[0] + e->vkick * orb.vec[2]);
        apply_energy_kick(phi, orb, ele.p);
      }
      break;
    case BMADGPU_SBEND: {
      // bend_edge_kick, fringe_mod.f90:40-128
      if (!fringe_here(ele, particle_at)) break;
      if (particle_at == first_track_edge) hard_multipole_edge_kick(ele, particle_at, orb);
      switch (e->fringe_type) {
        case BMADGPU_FRINGE_FULL:
          exact_bend_edge_kick(ele, particle_at, orb);
          break;
        case BMADGPU_FRINGE_BASIC_BEND: case BMADGPU_FRINGE_HARD_EDGE_ONLY:
          hwang_bend_edge_kick(ele, particle_at, orb, nullptr);
          break;
        default:
          return BMADGPU_EUNSUPPORTED;
      }
      if (particle_at == second_track_edge) hard_multipole_edge_kick(ele, particle_at, orb);
      break;
    }
    default:
      break;
  }
  if (particle_at == first_track_edge) electric_longitudinal_fringe(orb, ele, a_el, b_el, ix_elec_max, at_sign);
  return 0;
}

// init_fringe_info has_fringe, bmad/low_level/init_fringe_info.f90:22-55
bool has_fringe(const Ele& ele) {
  const bmadgpu_element* e = ele.e;
  switch (e->key) {
    case BMADGPU_RFCAVITY: case BMADGPU_ELSEPARATOR: return true;
    case BMADGPU_QUADRUPOLE: case BMADGPU_SBEND: case BMADGPU_SEXTUPOLE: case BMADGPU_OCTUPOLE:
    case BMADGPU_THICK_MULTIPOLE:
      if ((e->fringe_type == BMADGPU_FRINGE_NONE || e->fringe_at == BMADGPU_NO_END) && !ele.has_elec) return false;
      return true;
  }
  return false;
}

// ---------------------------------------------------------------------------------------------
// Element maps

qp element_t_update(const Coord& start, const Coord& orbit, const Ele& ele) {
  // orbit%t = start_orb%t + delta_ref_time + (start_orb%vec(5) - orbit%vec(5)) / (orbit%beta * c_light)
  return start.t + (qp)ele.e->delta_ref_time + (qp)((start.vec[4] - orbit.vec[4]) / (orbit.beta * c_light));
}

// track_a_quadrupole, bmad/low_level/track_a_quadrupole.f90
int track_a_quadrupole(Coord& orbit, const Ele& ele) {
  const bmadgpu_element* e = ele.e;
  Coord start_orb = orbit;
  double charge_dir = 1.0;
  double length = 1 * e->l;
  double an[n_pole_maxx + 1], bn[n_pole_maxx + 1], ane[n_pole_maxx + 1], bne[n_pole_maxx + 1], b1;
  int ix_mag_max, ix_elec_max, err;
  if ((err = multipole_ele_to_ab(ele, false, &ix_mag_max, an, bn, magnetic, true, &b1))) return err;
  if ((err = multipole_ele_to_ab(ele, false, &ix_elec_max, ane, bne, electric, false, nullptr))) return err;
  int n_step = 1;
  if (ix_mag_max > -1 || ix_elec_max > -1) n_step = std::max(nint(std::fabs(length) / ele.ds_step), 1);
  double r_step = 1.0 / n_step;
  double step_len = e->l * r_step;
  if (length == 0) n_step = 0;
  if (ele.has_misalign) {
    if ((err = offset_particle(ele, set_, orbit, true, false))) return err;
  }
  bool fr = has_fringe(ele);
  if (fr) {
    if ((err = apply_element_edge_kick(orbit, ele, first_track_edge))) return err;
    if (orbit.state != BMADGPU_ALIVE) return 0;
  }
  if (ix_mag_max > -1) ab_multipole_kicks(an, bn, ix_mag_max, ele, orbit, magnetic, r_step / 2);
  if (ix_elec_max > -1) ab_multipole_kicks(ane, bne, ix_elec_max, ele, orbit, electric, step_len / 2);
  for (int i = 1; i <= n_step; i++) {
    double rel_p = 1 + orbit.vec[5];
    double k1 = charge_dir * b1 / (length * rel_p);
    double mx[2][2], my[2][2], dz_x[3], dz_y[3];
    quad_mat2_calc(-k1, step_len, rel_p, mx, dz_x);
    quad_mat2_calc(k1, step_len, rel_p, my, dz_y);
    double* v = orbit.vec;
    v[4] = v[4] + (dz_x[0] * (v[0] * v[0]) + dz_x[1] * v[0] * v[1] + dz_x[2] * (v[1] * v[1]) +
                   dz_y[0] * (v[2] * v[2]) + dz_y[1] * v[2] * v[3] + dz_y[2] * (v[3] * v[3]));
    double x = v[0], px = v[1], y = v[2], py = v[3];
    v[0] = (0 + mx[0][0] * x) + mx[0][1] * px;
    v[1] = (0 + mx[1][0] * x) + mx[1][1] * px;
    v[2] = (0 + my[0][0] * y) + my[0][1] * py;
    v[3] = (0 + my[1][0] * y) + my[1][1] * py;
    v[4] = v[4] + low_energy_z_correction(orbit, ele, step_len);
    if (i == n_step) {
      if (ix_mag_max > -1) ab_multipole_kicks(an, bn, ix_mag_max, ele, orbit, magnetic, r_step / 2);
      if (ix_elec_max > -1) ab_multipole_kicks(ane, bne, ix_elec_max, ele, orbit, electric, step_len / 2);
    } else {
      if (ix_mag_max > -1) ab_multipole_kicks(an, bn, ix_mag_max, ele, orbit, magnetic, r_step);
      if (ix_elec_max > -1) ab_multipole_kicks(ane, bne, ix_elec_max, ele, orbit, electric, step_len);
    }
  }
  if (fr) {
    if ((err = apply_element_edge_kick(orbit, ele, second_track_edge))) return err;
    if (orbit.state != BMADGPU_ALIVE) return 0;
  }
  if (ele.has_misalign) {
    if ((err = offset_particle(ele, unset_, orbit, true, false))) return err;
  }
  orbit.t = element_t_update(start_orb, orbit, ele);
  return 0;
}

// track_this_elsep (contained in track_a_thick_multipole, track_a_thick_multipole.f90:137-240, no
// matrix): one step through the separator's transverse electric field, in the frame turned by
// angle_E; false if the particle was lost (on lost_pz the orbit returns to the element's start).
bool track_this_elsep(Coord& orbit, const Coord& start_orb, const Ele& ele, double step_len, double angle_E,
                      double k_E, double beta_ref) {
  const bmadgpu_param* p = ele.p;
  const double p0c = p->p0c, mc2 = p->mass;
  tilt_coords(angle_E, orbit.vec);
  const double beta = orbit.beta, px = orbit.vec[1], py = orbit.vec[3], pz = orbit.vec[5];
  const double pc = p0c * (1 + pz);
  const double E_tot = pc / beta;
  const double E_rel = E_tot / p0c;
  const double mr = mc2 / p0c;
  const double p_factor = mr * mr + px * px + py * py;
  if (E_rel * E_rel < p_factor) {
    orbit = start_orb;
    orbit.state = BMADGPU_LOST_PZ;
    return false;
  }
  const double ps2 = E_rel * E_rel - p_factor;
  const double ps = std::sqrt(ps2);
  const double coef = k_E * step_len / ps;
  if (std::fabs(coef) > 10) {
    orbit.state = BMADGPU_LOST;
    return false;
  }
  double sinh_k, cosh_k, cosh1_k;
  const double c2 = coef * coef, c4 = c2 * c2;
  if (std::fabs(coef) < 1e-3) {
    const double alpha = step_len / ps;
    sinh_k = alpha * (1 + c2 / 6 + c4 / 120);
    cosh1_k = alpha * coef * (1.0 / 2 + c2 / 24 + c4 / 720);
    cosh_k = lm.cosh(coef) / k_E;
  } else {
    cosh_k = lm.cosh(coef) / k_E;
    sinh_k = lm.sinh(coef) / k_E;
    cosh1_k = cosh_k - 1 / k_E;
  }
  const double dx = E_rel * cosh1_k + px * sinh_k;
  orbit.vec[0] = orbit.vec[0] + dx;
  orbit.vec[1] = k_E * (E_rel * sinh_k + px * cosh_k);
  orbit.vec[2] = orbit.vec[2] + step_len * py / ps;
  const double dct = E_rel * sinh_k + px * cosh1_k;
  orbit.vec[4] = orbit.vec[4] + orbit.beta * (step_len / beta_ref - dct);
  apply_energy_kick(dx * k_E * p0c, orbit, p);
  tilt_coords(-angle_E, orbit.vec);
  return true;
}

// track_a_thick_multipole, bmad/low_level/track_a_thick_multipole.f90:18-133
int track_a_thick_multipole(Coord& orbit, const Ele& ele) {
  const bmadgpu_element* e = ele.e;
  Coord start_orb = orbit;
  double length = e->l * 1;
  double an[n_pole_maxx + 1], bn[n_pole_maxx + 1], ane[n_pole_maxx + 1], bne[n_pole_maxx + 1];
  int ix_mag_max, ix_elec_max, err;
  // the separator's field (:49-65): strength k_E = kick / l along the angle atan2(vk, hk)
  double kick = 0, angle_E = 0, k_E = 0, beta_ref = 0;
  if (e->key == BMADGPU_ELSEPARATOR) {
    const double rtc = 1.0 * (ele.p->charge < 0 ? -1.0 : 1.0);  // |rel_tracking_charge| sign_of(charge)
    beta_ref = ele.p->p0c / ele.p->e_tot;
    const double hk = e->hkick * rtc, vk = e->vkick * rtc;
    kick = std::sqrt(hk * hk + vk * vk);
    angle_E = lm.atan2(vk, hk);
    k_E = (length == 0) ? 1.0 : kick / e->l;
  }
  if ((err = multipole_ele_to_ab(ele, false, &ix_mag_max, an, bn, magnetic, true, nullptr))) return err;
  if ((err = multipole_ele_to_ab(ele, false, &ix_elec_max, ane, bne, electric, false, nullptr))) return err;
  int n_step;
  if (kick == 0 && ix_mag_max == -1 && ix_elec_max == -1) n_step = 1;
  else n_step = std::max(nint(std::fabs(length / ele.ds_step)), 1);
  double r_step = 1.0 / n_step;
  double step_len = length / n_step;
  if (ele.has_misalign) {
    if ((err = offset_particle(ele, set_, orbit, true, false))) return err;
  }
  bool fr = has_fringe(ele);
  if (fr) {
    if ((err = apply_element_edge_kick(orbit, ele, first_track_edge))) return err;
    if (orbit.state != BMADGPU_ALIVE) return 0;
  }
  double ac_amp = 1;
  if (ix_mag_max > -1) ab_multipole_kicks(an, bn, ix_mag_max, ele, orbit, magnetic, ac_amp * r_step / 2);
  if (ix_elec_max > -1) ab_multipole_kicks(ane, bne, ix_elec_max, ele, orbit, electric, ac_amp * step_len / 2);
  for (int i = 1; i <= n_step; i++) {
    if (e->key == BMADGPU_ELSEPARATOR && kick != 0) {
      if (!track_this_elsep(orbit, start_orb, ele, step_len, angle_E, k_E, beta_ref)) return 0;
    } else {
      track_a_drift(orbit, step_len, ele.p);
    }
    if (i == n_step) {
      if (ix_mag_max > -1) ab_multipole_kicks(an, bn, ix_mag_max, ele, orbit, magnetic, ac_amp * r_step / 2);
      if (ix_elec_max > -1) ab_multipole_kicks(ane, bne, ix_elec_max, ele, orbit, electric, ac_amp * step_len / 2);
    } else {
      if (ix_mag_max > -1) ab_multipole_kicks(an, bn, ix_mag_max, ele, orbit, magnetic, ac_amp * r_step);
      if (ix_elec_max > -1) ab_multipole_kicks(ane, bne, ix_elec_max, ele, orbit, electric, ac_amp * step_len);
    }
  }
  if (fr) {
    if ((err = apply_element_edge_kick(orbit, ele, second_track_edge))) return err;
    if (orbit.state != BMADGPU_ALIVE) return 0;
  }
  if (ele.has_misalign) {
    if ((err = offset_particle(ele, unset_, orbit, true, false))) return err;
  }
  orbit.t = element_t_update(start_orb, orbit, ele);
  return 0;
}

// sbend_body_with_k1_map, bmad/low_level/track_a_bend.f90:500-659 (no matrix)
void sbend_body_with_k1_map(const Ele& ele, double dg, double b1, int n_step, Coord& orbit) {
  const bmadgpu_element* e = ele.e;
  double rel_charge_dir = 1.0;
  double g = e->g;
  double length = 1 * e->l / n_step;
  double k1 = b1 / e->l;
  double g_tot = (g + dg) * rel_charge_dir;
  double rel_p = (1 + orbit.vec[5]);
  double rel_p2 = rel_p * rel_p;
  double k_x = k1 + g * g_tot;
  double x_c = (g * rel_p - g_tot) / k_x;
  double om_x = std::sqrt(std::fabs(k_x) / rel_p);
  double om_y = std::sqrt(std::fabs(k1) / rel_p);
  double tau_x = -std::copysign(1.0, k_x);
  double tau_y = std::copysign(1.0, k1);
  double s_x, c_x, z2, s_y, c_y;
  double arg = om_x * length;
  if (arg < 1e-6) {
    s_x = (1 + tau_x * (arg * arg) / 6) * length;
    c_x = 1 + tau_x * (arg * arg) / 2;
    z2 = g * (length * length) / (2 * rel_p);
  } else if (k_x > 0) {
    s_x = lm.sin(arg) / om_x;
    c_x = lm.cos(arg);
    z2 = tau_x * g * (1 - c_x) / (rel_p * (om_x * om_x));
  } else {
    s_x = lm.sinh(arg) / om_x;
    c_x = lm.cosh(arg);
    z2 = tau_x * g * (1 - c_x) / (rel_p * (om_x * om_x));
  }
  arg = om_y * length;
  if (arg < 1e-6) {
    s_y = (1 + tau_y * (arg * arg) / 6) * length;
    c_y = 1 + tau_y * (arg * arg) / 2;
  } else if (k1 < 0) {
    s_y = lm.sin(om_y * length) / om_y;
    c_y = lm.cos(om_y * length);
  } else {
    s_y = lm.sinh(om_y * length) / om_y;
    c_y = lm.cosh(om_y * length);
  }
  double r[6];
  for (int i = 0; i < 6; i++) r[i] = orbit.vec[i];
  r[0] = r[0] - x_c;
  double z0 = -g * x_c * length;
  double z1 = -g * s_x;
  double z11 = tau_x * (om_x * om_x) * (length - c_x * s_x) / 4;
  double z12 = -tau_x * (om_x * om_x) * (s_x * s_x) / (2 * rel_p);
  double z22 = -(length + c_x * s_x) / (4 * rel_p2);
  double z33 = tau_y * (om_y * om_y) * (length - c_y * s_y) / 4;
  double z34 = -tau_y * (om_y * om_y) * (s_y * s_y) / (2 * rel_p);
  double z44 = -(length + c_y * s_y) / (4 * rel_p2);
  orbit.vec[0] = c_x * r[0] + s_x * r[1] / rel_p + x_c;
  orbit.vec[1] = tau_x * (om_x * om_x) * rel_p * s_x * r[0] + c_x * r[1];
  orbit.vec[2] = c_y * r[2] + s_y * r[3] / rel_p;
  orbit.vec[3] = tau_y * (om_y * om_y) * rel_p * s_y * r[2] + c_y * r[3];
  orbit.vec[4] = r[4] + 1 * 1 * z0 + z1 * r[0] + z2 * r[1] + z11 * (r[0] * r[0]) + z12 * r[0] * r[1] +
                 z22 * (r[1] * r[1]) + z33 * (r[2] * r[2]) + z34 * r[2] * r[3] + z44 * (r[3] * r[3]);
}

// elec_multipole_field, bmad/code/elec_multipole_field.f90:25-60 (field only, no derivatives)
void elec_multipole_field(double a, double b, int n, const Coord& coord, double* Ex, double* Ey) {
  *Ex = 0;
  *Ey = 0;
  if (a == 0 && b == 0) return;
  double x = coord.vec[0], y = coord.vec[2];
  for (int m = 0; m <= n; m += 2) {
    double f = cm.no_n_fact(n, m) * mexp(x, n - m) * mexp(y, m);
    *Ex = *Ex - b * f;
    *Ey = *Ey - a * f;
  }
  for (int m = 1; m <= n; m += 2) {
    double f = cm.no_n_fact(n, m) * mexp(x, n - m) * mexp(y, m);
    *Ex = *Ex + a * f;
    *Ey = *Ey - b * f;
  }
}

// apply_multipole_kicks (contained in track_a_bend), track_a_bend.f90:338-471, exact_multipoles
// = off: the fields of both kinds from the incoming orbit, then the magnetic kick, then the
// electric kick with its energy change.
void bend_apply_multipole_kicks(const Ele& ele, double coef, double step_len, double r_step, int ix_mag_max,
                                const double* an, const double* bn, int ix_elec_max, const double* ane,
                                const double* bne, Coord& orbit) {
  const bmadgpu_element* e = ele.e;
  const bmadgpu_param* p = ele.p;
  double B1 = 0, B2 = 0, E1 = 0, E2 = 0;
  double f_p0c = r_step * p->p0c / (c_light * p->charge);
  for (int i = 0; i <= ix_mag_max; i++) {
    if (an[i] == 0 && bn[i] == 0) continue;
    double kx, ky;
    ab_multipole_kick(an[i], bn[i], i, 0, orbit, p, &kx, &ky, magnetic, 0, false);
    B1 = B1 + f_p0c * ky;
    B2 = B2 - f_p0c * kx;
  }
  for (int i = 0; i <= ix_elec_max; i++) {
    if (ane[i] == 0 && bne[i] == 0) continue;
    double ex, ey;
    elec_multipole_field(ane[i], bne[i], i, orbit, &ex, &ey);
    E1 = E1 + ex;
    E2 = E2 + ey;
  }
  if (ix_mag_max > -1) {
    double c_dir = 1.0 * p->charge;  // orientation * direction * charge_of(species)
    double f_coef = coef * c_dir * (1 + e->g * orbit.vec[0]) * c_light / orbit.p0c;
    orbit.vec[1] = orbit.vec[1] - f_coef * B2;
    orbit.vec[3] = orbit.vec[3] + f_coef * B1;
  }
  if (ix_elec_max > -1) {
    Coord orb0 = orbit;
    double rel_p0 = 1 + orb0.vec[5];
    double ps2 = rel_p0 * rel_p0 - orb0.vec[1] * orb0.vec[1] - orb0.vec[3] * orb0.vec[3];
    double ps = std::sqrt(ps2) / rel_p0;
    double f_coef = step_len * coef * (1 + e->g * orb0.vec[0]) * p->charge / (ps * orb0.beta * orb0.p0c);
    double kx = f_coef * E1, ky = f_coef * E2;
    double alpha = (kx * (2 * orb0.vec[1] + kx) + ky * (2 * orb0.vec[3] + ky)) / (rel_p0 * rel_p0);
    orbit.vec[1] = orb0.vec[1] + kx;
    orbit.vec[3] = orb0.vec[3] + ky;
    orbit.vec[5] = orb0.vec[5] + rel_p0 * sqrt_one(alpha);
    double mp = p->mass / orbit.p0c;
    orbit.beta = (1 + orbit.vec[5]) /
                 std::sqrt(ps2 + orbit.vec[1] * orbit.vec[1] + orbit.vec[3] * orbit.vec[3] + mp * mp);
    orbit.vec[4] = orb0.vec[4] * orbit.beta / orb0.beta;
  }
}

// track_a_bend, bmad/low_level/track_a_bend.f90:18-333
int track_a_bend(Coord& orbit, const Ele& ele) {
  const bmadgpu_element* e = ele.e;
  const bmadgpu_param* p = ele.p;
  Coord start_orb = orbit;
  int err;
  if (ele.has_misalign) {
    if ((err = offset_particle(ele, set_, orbit, true, false))) return err;
  }
  double rel_charge_dir = 1.0;
  if ((err = apply_element_edge_kick(orbit, ele, first_track_edge))) return err;
  if (orbit_too_large(orbit, p)) return 0;
  if (e->exact_multipoles != 0 && e->exact_multipoles != 1) return BMADGPU_EUNSUPPORTED;
  double an[n_pole_maxx + 1], bn[n_pole_maxx + 1], ane[n_pole_maxx + 1], bne[n_pole_maxx + 1], b1;
  int ix_mag_max, ix_elec_max;
  if ((err = multipole_ele_to_ab(ele, false, &ix_mag_max, an, bn, magnetic, true, &b1))) return err;
  b1 = b1 * rel_charge_dir;
  if (std::fabs(b1) < 1e-10) {
    bn[1] = b1;
    b1 = 0;
  }
  if ((err = multipole_ele_to_ab(ele, false, &ix_elec_max, ane, bne, electric, false, nullptr))) return err;
  double length = 1 * e->l;
  double g = e->g, dg;
  if (length == 0) {
    dg = 0;
  } else {
    dg = bn[0] / e->l;
    bn[0] = 0;
  }
  double g_tot = (g + dg) * rel_charge_dir;
  if (!e->is_on) {
    dg = -g;
    g_tot = 0;
    b1 = 0;
  }
  int n_step = 1;
  if (ix_mag_max > -1 || ix_elec_max > -1) n_step = std::max(nint(std::fabs(length) / ele.ds_step), 1);
  double r_step = 1.0 / n_step;
  double step_len = length / n_step;
  double angle = g * step_len;
  const bool kicks = ix_mag_max > -1 || ix_elec_max > -1;
  if (kicks) bend_apply_multipole_kicks(ele, 0.5, step_len, r_step, ix_mag_max, an, bn, ix_elec_max, ane, bne, orbit);
  for (int n = 1; n <= n_step; n++) {
    if (b1 != 0) {
      sbend_body_with_k1_map(ele, dg, b1, n_step, orbit);
      orbit.vec[4] = orbit.vec[4] + low_energy_z_correction(orbit, ele, step_len);
    } else if ((g == 0 && dg == 0) || step_len == 0) {
      track_a_drift(orbit, step_len, p);
    } else {
      double x = orbit.vec[0], px = orbit.vec[1], y = orbit.vec[2], py = orbit.vec[3];
      double z = orbit.vec[4], pz = orbit.vec[5];
      double rel_p = 1 + pz;
      double rel_p2 = rel_p * rel_p;
      if (dg == 0 && std::fabs(x * g) < 1e-9 && std::fabs(px) < 1e-9 && std::fabs(py) < 1e-9 &&
          std::fabs(pz) < 1e-9) {
        double ll = step_len;
        double cos_a = lm.cos(angle), sin_a = lm.sin(angle);
        double sinc_a = sinc(angle), cosc_a = cosc(angle);
        double m2 = p->mass * p->mass;
        double rpp = rel_p * orbit.p0c;
        double gam2 = m2 / (rpp * rpp + m2);
        double gl = g * ll;
        double m56 = ll * (gam2 - (gl * gl) * sincc(angle));
        orbit.vec[0] = cos_a * x + ll * sinc_a * px + g * (ll * ll) * cosc_a * pz;
        orbit.vec[1] = -g * sin_a * x + cos_a * px + g * ll * sinc_a * pz;
        orbit.vec[2] = y + ll * py;
        orbit.vec[4] = -g * ll * sinc_a * x - g * (ll * ll) * cosc_a * px + z + m56 * pz;
      } else {
        double beta_ref = p->p0c / p->e_tot;
        double sinc_a = sinc(angle);
        double pt = std::sqrt(rel_p2 - py * py);
        if (std::fabs(px) > pt) {
          orbit.state = BMADGPU_LOST_PZ;
          return 0;
        }
        double g_p = g_tot / pt;
        double phi_1 = lm.asin(px / pt);
        double cos_a = lm.cos(angle), sin_a = lm.sin(angle);
        double cosc_a = cosc(angle);
        double cos_plus = lm.cos(angle + phi_1);
        double sin_plus = lm.sin(angle + phi_1);
        double gx1 = 1 + g * x;
        double ls = gx1 * step_len * sinc_a;
        double alpha = 2 * gx1 * sin_plus * step_len * sinc_a - g_p * (ls * ls);
        double r = cos_plus * cos_plus + g_p * alpha;
        if (r < 0 || (std::fabs(g_p) < 1e-5 && std::fabs(cos_plus) < 1e-5)) {
          orbit.state = BMADGPU_LOST;
          orbit.vec[0] = 2 * p->max_aperture_limit;
          return 0;
        }
        double rad = std::sqrt(r);
        double denom, xi;
        if (cos_plus > 0) {
          denom = rad + cos_plus;
          xi = alpha / denom;
        } else {
          denom = rad - cos_plus;
          xi = denom / g_p;
        }
        orbit.vec[0] = x * cos_a - (step_len * step_len) * g * cosc_a + xi;
        if (std::fabs(orbit.vec[0]) > p->max_aperture_limit) {
          orbit.state = BMADGPU_LOST;
          return 0;
        }
        double L_u = xi;
        double L_v = -1 * (step_len * sinc_a + x * sin_a);
        double L_c = std::sqrt(L_v * L_v + L_u * L_u);
        double angle_p = 2 * (angle + phi_1 - 1 * lm.atan2(L_u, -L_v));
        double L_p = 1 * L_c / sinc(angle_p / 2);
        orbit.vec[1] = pt * lm.sin(phi_1 + angle - angle_p);
        orbit.vec[2] = y + py * L_p / pt;
        orbit.vec[4] = z + orbit.beta * step_len / beta_ref - rel_p * L_p / pt;
      }
    }
    if (kicks) {
      double c = (n == n_step) ? 0.5 : 1.0;
      bend_apply_multipole_kicks(ele, c, step_len, r_step, ix_mag_max, an, bn, ix_elec_max, ane, bne, orbit);
    }
  }
  if (orbit_too_large(orbit, p)) return 0;
  if ((err = apply_element_edge_kick(orbit, ele, second_track_edge))) return err;
  if (ele.has_misalign) {
    if ((err = offset_particle(ele, unset_, orbit, true, false))) return err;
  }
  orbit.t = element_t_update(start_orb, orbit, ele);
  orbit.s = ele.s;
  return 0;
}

// track_a_rfcavity, bmad/low_level/track_a_rfcavity.f90:17-146 (relative time tracking)
int track_a_rfcavity(Coord& orbit, const Ele& ele) {
  const bmadgpu_element* e = ele.e;
  const bmadgpu_param* p = ele.p;
  if (e->rf_frequency == 0 && e->voltage != 0) {
    orbit.state = BMADGPU_LOST;
    return 0;
  }
  double length = e->l * 1;
  int n_step = 1;
  double r_step = 1.0 / n_step;
  double step_len = length / n_step;
  int n_slice = std::max(1, nint(std::fabs(length) / ele.ds_step));
  double charge_dir = 1.0;
  double an[n_pole_maxx + 1], bn[n_pole_maxx + 1], ane[n_pole_maxx + 1], bne[n_pole_maxx + 1];
  int ix_mag_max, ix_elec_max, err;
  if ((err = multipole_ele_to_ab(ele, false, &ix_mag_max, an, bn, magnetic, true, nullptr))) return err;
  if ((err = multipole_ele_to_ab(ele, false, &ix_elec_max, ane, bne, electric, false, nullptr))) return err;
  if ((err = offset_particle(ele, set_, orbit, true, true))) return err;
  if (ix_mag_max > -1) ab_multipole_kicks(an, bn, ix_mag_max, ele, orbit, magnetic, 0.5 * r_step);
  if (ix_elec_max > -1) ab_multipole_kicks(ane, bne, ix_elec_max, ele, orbit, electric, 0.5 * step_len);
  double voltage = (e->is_on ? e->voltage : 0.0) * charge_dir;  // e_accel_field(ele, voltage$, .true.)
  // particle_rf_time (particle_rf_time.f90:32-120): relative time -z/(beta c), real(qp),
  // folded with modulo2(time, 0.5/rf_freq) in qp.
  qp time = (qp)(-orbit.vec[4] / (orbit.beta * c_light));
  qp f_q = (qp)e->rf_frequency;
  if (e->rf_frequency != 0) time = modulo2q(time, (qp)0.5 / f_q);
  qp ph_q = (qp)twopi * ((qp)e->phi0 - (time - (qp)0.0) * f_q);
  double phase0 = (double)ph_q;
  phase0 = phase0 + twopi * e->phi0_multipass;
  double phase = modulo2(phase0, pi);
  // rf_coupler_kick: coupler_strength = 0 on the path -> no kick
  for (int i = 0; i <= n_slice; i++) {
    double dE = 1 * voltage * lm.sin(phase) / n_slice;
    if (i == 0 || i == n_slice) dE = dE / 2;
    apply_energy_kick(dE, orbit, p);
    if (orbit.vec[5] == -1) {
      orbit.state = BMADGPU_LOST_PZ;
      return 0;
    }
    if (i != n_slice) {
      double z = orbit.vec[4];
      track_a_drift(orbit, length / n_slice, p);
      phase = phase + twopi * e->rf_frequency * (orbit.vec[4] - z) / (c_light * orbit.beta);
    }
  }
  orbit.phase1 = modulo2(phase, 0.5);
  if (ix_elec_max > -1) ab_multipole_kicks(ane, bne, ix_elec_max, ele, orbit, electric, 0.5 * step_len);
  if (ix_mag_max > -1) ab_multipole_kicks(an, bn, ix_mag_max, ele, orbit, magnetic, 0.5 * r_step);
  if ((err = offset_particle(ele, unset_, orbit, true, true))) return err;
  return 0;
}

// thin multipole / ab_multipole branch of track1_bmad, bmad/low_level/track1_bmad.f90:142-166
int track_thin_multipole(Coord& orbit, const Ele& ele) {
  int err;
  if (ele.has_misalign) {
    if ((err = offset_particle(ele, set_, orbit, false, true))) return err;
  }
  double knl[n_pole_maxx + 1], tilt[n_pole_maxx + 1];
  int ix_pole_max;
  if ((err = multipole_ele_to_kt(ele, true, &ix_pole_max, knl, tilt, magnetic, false))) return err;
  if (ix_pole_max > -1) {
    bool ref_orb_offset = (ele.e->key == BMADGPU_MULTIPOLE);
    for (int n = 0; n <= n_pole_maxx; n++) {
      if (knl[n] == 0) continue;
      multipole_kick(knl[n], tilt[n], n, orbit, ref_orb_offset);
    }
  }
  if (ele.has_misalign) {
    if ((err = offset_particle(ele, unset_, orbit, false, true))) return err;
  }
  return 0;
}

// track1_bmad, bmad/low_level/track1_bmad.f90:22-283
int track1_bmad(Coord& orbit, const Ele& ele) {
  const bmadgpu_element* e = ele.e;
  int key = e->key;
  if (!e->is_on) {
    switch (key) {
      case BMADGPU_AB_MULTIPOLE: case BMADGPU_MULTIPOLE: key = -1; break;
      case BMADGPU_SBEND: break;
      default: key = BMADGPU_DRIFT;
    }
  }
  int err = 0;
  switch (key) {
    case -1: break;
    case BMADGPU_DRIFT: track_a_drift(orbit, e->l * 1, ele.p); break;
    case BMADGPU_MONITOR: case BMADGPU_INSTRUMENT: case BMADGPU_PIPE:
    case BMADGPU_RCOLLIMATOR: case BMADGPU_ECOLLIMATOR:  // track1_bmad.f90:87-88
    case BMADGPU_KICKER: case BMADGPU_HKICKER: case BMADGPU_VKICKER: case BMADGPU_ELSEPARATOR:
    case BMADGPU_OCTUPOLE: case BMADGPU_THICK_MULTIPOLE: case BMADGPU_SEXTUPOLE:
      err = track_a_thick_multipole(orbit, ele);
      break;
    case BMADGPU_MARKER: orbit.t = orbit.t + (qp)e->delta_ref_time; break;
    case BMADGPU_MULTIPOLE: case BMADGPU_AB_MULTIPOLE: err = track_thin_multipole(orbit, ele); break;
    case BMADGPU_QUADRUPOLE: err = track_a_quadrupole(orbit, ele); break;
    case BMADGPU_RFCAVITY: err = track_a_rfcavity(orbit, ele); break;
    case BMADGPU_SBEND: err = track_a_bend(orbit, ele); break;
    default: return BMADGPU_EUNSUPPORTED;
  }
  if (err) return err;
  orbit.s = ele.s;
  return 0;
}

// ---------------------------------------------------------------------------------------------
// Bookkeeping

// check_bend, forest/code/So_fitting.f90:3516-3548
void check_bend(double xl, double ggi, double rhoi, double xbend1, double gf[8], int* met) {
  double gg = (double)(long long)ggi;
  if (gg == 0.0) gg = 1.0;
  double co[8] = {0, 0, 1.0 / 12.0, 0, 0.17, 0, 0.17e-1, 0};
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

bool any_nonzero(const double* a, int n) {
  for (int i = 0; i < n; i++) if (a[i] != 0) return true;
  return false;
}

// attribute_bookkeeper.f90:146-170 (tilt_tot, has_misalign) and :292-400 (ds_step, num_steps)
int make_ele(const bmadgpu_element* e, const bmadgpu_param* p, int ix_ele, Ele& ele) {
  ele.e = e;
  ele.p = p;
  ele.ix_ele = ix_ele;
  ele.s_start = 0;
  ele.s = e->l;
  ele.has_elec = any_nonzero(e->a_pole_elec, BMADGPU_N_POLE) || any_nonzero(e->b_pole_elec, BMADGPU_N_POLE);
  ele.has_mag = any_nonzero(e->a_pole, BMADGPU_N_POLE) || any_nonzero(e->b_pole, BMADGPU_N_POLE);
  if (e->orientation != 1 && e->orientation != 0) return BMADGPU_EUNSUPPORTED;
  if (e->key == BMADGPU_MULTIPOLE && ele.has_elec) return BMADGPU_EUNSUPPORTED;  // skew ksl_pole
  if (e->key == BMADGPU_SBEND) {
    ele.tilt_tot = 0;
    ele.ref_tilt_tot = e->ref_tilt;
    ele.has_misalign = (e->ref_tilt != 0 || e->roll != 0);
    if (e->tilt != 0) return BMADGPU_EUNSUPPORTED;
  } else {
    ele.tilt_tot = e->tilt;
    ele.ref_tilt_tot = 0;
    ele.has_misalign = (e->tilt != 0);
  }
  ele.has_misalign = ele.has_misalign || e->x_offset != 0 || e->y_offset != 0 || e->z_offset != 0 ||
                     e->x_pitch != 0 || e->y_pitch != 0;
  double ds_step = e->ds_step;
  double num_steps = e->num_steps;
  if (num_steps == 0 && e->key == BMADGPU_RFCAVITY) num_steps = 10;  // set_ele_defaults.f90:319
  double L = e->l;
  if (ds_step == 0 && num_steps == 0) {
    switch (e->key) {
      case BMADGPU_DRIFT: case BMADGPU_PIPE: case BMADGPU_INSTRUMENT: case BMADGPU_MONITOR:
      case BMADGPU_RCOLLIMATOR: case BMADGPU_ECOLLIMATOR:
        num_steps = 1;
        ds_step = L;
        break;
      case BMADGPU_SBEND: case BMADGPU_QUADRUPOLE: case BMADGPU_SEXTUPOLE:
        if (L != 0) {
          double knl[n_pole_maxx + 1], tilt[n_pole_maxx + 1];
          int ix;
          int err = multipole_ele_to_kt(ele, false, &ix, knl, tilt, magnetic, true);
          if (err) return err;
          for (int i = 0; i <= n_pole_maxx; i++) knl[i] = std::fabs(knl[i]);
          double bend_factor = knl[0] / L;
          double radius0 = e->r0_mag;
          if (radius0 == 0) radius0 = 0.01;
          double quad_factor = 0;
          if (e->key == BMADGPU_SBEND) {
            bend_factor = bend_factor + std::max(std::fabs(e->g), std::fabs(e->g + e->dg));
            quad_factor = knl[1] + knl[2] * radius0 + L * (bend_factor * bend_factor);
          } else if (e->key == BMADGPU_QUADRUPOLE) {
            quad_factor = 50 * (knl[1] + L * (bend_factor * bend_factor));
          } else {
            quad_factor = knl[2] * radius0 + L * (bend_factor * bend_factor);
          }
          if (ele.has_elec) {
            double r0e = e->r0_elec;
            if (r0e == 0) r0e = 0.01;
            double a[n_pole_maxx + 1], b[n_pole_maxx + 1];
            int ixp;
            multipole_ele_to_ab(ele, false, &ixp, a, b, electric, false, nullptr);
            bend_factor = bend_factor + (std::fabs(a[0]) + std::fabs(b[0])) / p->p0c;
            quad_factor = quad_factor + (std::fabs(a[1]) + std::fabs(b[1]) + r0e * (std::fabs(a[2]) + std::fabs(b[2]))) / p->p0c;
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
    if (num_steps <= 0 || std::fabs(L) == 0) ds_step = p->default_ds_step;
    else ds_step = std::fabs(L) / num_steps;
  }
  ele.ds_step = ds_step;
  ele.num_steps = std::max(1, nint(std::fabs(L / ds_step)));
  return 0;
}

qp coord_tq(const oracle_coord* c) {
  qp t;
  std::memcpy(&t, c->t_qp, sizeof(qp));
  return t;
}

void to_internal(const oracle_coord* c, Coord& o) {
  for (int i = 0; i < 6; i++) o.vec[i] = c->vec[i];
  o.beta = c->beta;
  o.p0c = c->p0c;
  o.s = c->s;
  o.phase1 = c->phase1;
  o.t = coord_tq(c);
  o.state = c->state;
  o.location = c->location;
  o.ix_ele = c->ix_ele;
}

void to_external(const Coord& o, oracle_coord* c) {
  for (int i = 0; i < 6; i++) c->vec[i] = o.vec[i];
  c->beta = o.beta;
  c->p0c = o.p0c;
  c->s = o.s;
  c->phase1 = o.phase1;
  c->t = (double)o.t;
  std::memcpy(c->t_qp, &o.t, sizeof(qp));
  c->state = o.state;
  c->location = o.location;
  c->ix_ele = o.ix_ele;
}

// track1, bmad/code/track1.f90:44-343 (no radiation, spin, space charge or hooks)
int track1(Coord& orb, const Ele& ele) {
  orb.location = BMADGPU_UPSTREAM_END;
  orb.s = ele.s_start;
  orb.ix_ele = ele.ix_ele;
  if (orb.state != BMADGPU_ALIVE) return 0;
  int err = check_aperture_limit(orb, ele, first_track_edge);
  if (err) return err;
  if (orb.state != BMADGPU_ALIVE) return 0;
  err = track1_bmad(orb, ele);
  if (err) return err;
  if (orbit_too_large(orb, ele.p)) return 0;
  if (orb.state != BMADGPU_ALIVE) orb.location = BMADGPU_INSIDE;
  else orb.location = BMADGPU_DOWNSTREAM_END;
  if (orb.state != BMADGPU_ALIVE) return 0;
  return check_aperture_limit(orb, ele, second_track_edge);
}

int check_param(const bmadgpu_param* p) {
  if (!p) return BMADGPU_EINVAL;
  if (p->absolute_time_tracking || p->radiation_on) return BMADGPU_EUNSUPPORTED;
  return 0;
}

}  // namespace

// =============================================================================================
extern "C" {

int32_t oracle_element_num_steps(const bmadgpu_element* e, const bmadgpu_param* p) {
  Ele ele;
  int err = make_ele(e, p, 0, ele);
  if (err) return err;
  return ele.num_steps;
}

void oracle_init_coord(oracle_coord* orb, const double vec[6], const bmadgpu_param* p) {
  std::memset(orb, 0, sizeof(*orb));
  for (int i = 0; i < 6; i++) orb->vec[i] = vec[i];
  orb->p0c = p->p0c;
  if (orb->vec[5] == 0) {
    orb->beta = p->p0c / p->e_tot;
  } else {
    double pc = p->p0c * (1 + orb->vec[5]);
    orb->beta = pc / std::sqrt(pc * pc + p->mass * p->mass);
  }
  qp t = (qp)0 - (qp)(orb->vec[4] / (orb->beta * c_light));
  std::memcpy(orb->t_qp, &t, sizeof(qp));
  orb->t = (double)t;
  orb->state = BMADGPU_ALIVE;
  orb->location = BMADGPU_UPSTREAM_END;
  orb->direction = 1;
  orb->time_dir = 1;
}

int oracle_track1(oracle_coord* c, const bmadgpu_element* e, int32_t ix_ele, const bmadgpu_param* p) {
  int err = check_param(p);
  if (err) return err;
  Ele ele;
  if ((err = make_ele(e, p, ix_ele, ele))) return err;
  Coord o;
  to_internal(c, o);
  err = track1(o, ele);
  to_external(o, c);
  return err;
}

int oracle_hwang_bend_edge_kick(const bmadgpu_element* e, const bmadgpu_param* p, int32_t particle_at,
                                oracle_coord* c, double* mat6) {
  Ele ele;
  int err = make_ele(e, p, 0, ele);
  if (err) return err;
  Coord o;
  to_internal(c, o);
  hwang_bend_edge_kick(ele, particle_at, o, mat6);
  to_external(o, c);
  return 0;
}

int oracle_offset_particle(const bmadgpu_element* e, const bmadgpu_param* p, int32_t set, oracle_coord* c) {
  Ele ele;
  int err = make_ele(e, p, 0, ele);
  if (err) return err;
  Coord o;
  to_internal(c, o);
  err = offset_particle(ele, set ? set_ : unset_, o, true, true);
  to_external(o, c);
  return err;
}

int oracle_check_aperture(const bmadgpu_element* e, const bmadgpu_param* p, int32_t particle_at, oracle_coord* c,
                          double* unstable_factor) {
  Ele ele;
  int err = make_ele(e, p, 0, ele);
  if (err) return err;
  Coord o;
  to_internal(c, o);
  err = check_aperture_limit(o, ele, particle_at, unstable_factor);
  to_external(o, c);
  return err;
}

void oracle_set_libm(double (*f_sin)(double), double (*f_cos)(double), double (*f_asin)(double),
                     double (*f_atan2)(double, double), double (*f_sinh)(double), double (*f_cosh)(double),
                     double (*f_exp)(double), double (*f_tan)(double)) {
  if (!f_sin || !f_cos || !f_asin || !f_atan2 || !f_sinh || !f_cosh || !f_exp || !f_tan) {
    lm = Libm{h_sin, h_cos, h_asin, h_atan2, h_sinh, h_cosh, h_exp, h_tan};
    return;
  }
  lm = Libm{f_sin, f_cos, f_asin, f_atan2, f_sinh, f_cosh, f_exp, f_tan};
}

int32_t oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int oracle_track_ring(const bmadgpu_element* eles, int32_t n_ele, const bmadgpu_param* p,
                      bmadgpu_bunch* bunch, int32_t turn0, int32_t n_turns, int32_t n_threads,
                      double* moments) {
  int err = check_param(p);
  if (err) return err;
  if (!eles || !bunch || n_ele <= 0 || n_turns < 0 || bunch->n < 0) return BMADGPU_EINVAL;
  std::vector<Ele> ele(n_ele);
  for (int i = 0; i < n_ele; i++)
    if ((err = make_ele(&eles[i], p, i, ele[i]))) return err;
  const int64_t n = bunch->n;
  std::vector<Coord> part(n);
  for (int64_t j = 0; j < n; j++) {
    Coord& o = part[j];
    for (int i = 0; i < 6; i++) o.vec[i] = bunch->vec[i * n + j];
    o.beta = bunch->beta[j];
    o.p0c = p->p0c;
    o.s = 0;
    o.phase1 = 0;
    o.t = bunch->t ? (qp)bunch->t[j] : (qp)0;
    o.state = bunch->state[j];
    o.location = bunch->location ? bunch->location[j] : BMADGPU_UPSTREAM_END;
    o.ix_ele = bunch->ix_ele ? bunch->ix_ele[j] : -1;
  }
  int nt = n_threads > 0 ? n_threads : oracle_max_threads();
  std::vector<int32_t> lost_turn(n, -1);
  int fail = 0;
  for (int it = 0; it < n_turns && !fail; it++) {
    for (int ie = 0; ie < n_ele && !fail; ie++) {
      const Ele& el = ele[ie];
      // track1_bunch_hom particle loop, beam_utils.f90:81-86
#pragma omp parallel for num_threads(nt) schedule(static)
      for (int64_t j = 0; j < n; j++) {
        Coord& o = part[j];
        if (o.state != BMADGPU_ALIVE) continue;
        int e2 = track1(o, el);
        if (e2) {
#pragma omp atomic write
          fail = e2;
        }
        if (o.state != BMADGPU_ALIVE) lost_turn[j] = turn0 + it;
      }
    }
    if (moments) {
      double* m = moments + (int64_t)it * BMADGPU_N_MOMENTS;
      for (int k = 0; k < BMADGPU_N_MOMENTS; k++) m[k] = 0;
      for (int64_t j = 0; j < n; j++) {
        const Coord& o = part[j];
        if (o.state != BMADGPU_ALIVE) continue;
        m[0] += 1;
        int k = 7;
        for (int a = 0; a < 6; a++) {
          m[1 + a] += o.vec[a];
          for (int b = a; b < 6; b++) m[k++] += o.vec[a] * o.vec[b];
        }
      }
    }
  }
  if (fail) return fail;
  for (int64_t j = 0; j < n; j++) {
    const Coord& o = part[j];
    for (int i = 0; i < 6; i++) bunch->vec[i * n + j] = o.vec[i];
    bunch->beta[j] = o.beta;
    if (bunch->t) bunch->t[j] = (double)o.t;
    if (o.state != bunch->state[j] && lost_turn[j] >= 0) {
      if (bunch->ix_ele) bunch->ix_ele[j] = o.ix_ele;
      if (bunch->ix_turn) bunch->ix_turn[j] = lost_turn[j];
      if (bunch->location) bunch->location[j] = o.location;
    }
    bunch->state[j] = o.state;
  }
  return 0;
}

}  // extern "C"
