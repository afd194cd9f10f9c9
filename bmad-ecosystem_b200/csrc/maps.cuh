// maps.cuh -- FP64 device maps of Bmad's bmad_standard tracking, one particle per thread.
//
// Each function restates one reference routine (cited) on a particle held in registers, with
// the reference's operand order: in long-term tracking, rounding that differs systematically
// from the reference (a product regrouped around near-constant factors rounds the same way for
// every particle and every element) accumulates coherently turn after turn. Element invariants
// that the reference recomputes from element attributes alone come precomputed from the packed
// table with the same expressions, hence bit-identical. Functions of pz alone that the reference
// recomputes per element with the same expression are cached in the particle (refresh()).
// The kernels are compiled without FMA contraction, so the device results differ from the
// reference's only through the six transcendentals the maps call (sin, cos, asin, atan2, sinh,
// cosh). The library is built twice from this source: with the device libm (libbmadgpu.so, the
// fast build), and with BG_CR_MATH, where those six are correctly rounded (crmath.cuh) and the
// results are bit for bit those of the reference's algorithm run with a correctly rounded libm
// (libbmadgpu_cr.so).
#pragma once
#include <math.h>
#include <stdint.h>

#include "table.h"

// The maps' transcendentals: correctly rounded with BG_CR_MATH (device, or the test-only host
// build made with it), otherwise the device's or host's libm.
#if defined(BG_CR_MATH)
#include "crmath.cuh"
#define BG_CR_TRANSCENDENTALS 1
#endif

// The maps compile for the device (the product) and, for the test-only host check build
// (hostcheck.cpp: op counting and algorithm checks on CPU), for the host.
#if defined(__CUDACC__)
#define BG_HD __device__ __forceinline__
#define BG_COLD static __device__ __noinline__   // rare forms: one out-of-line copy
#else
#define BG_HD inline
#define BG_COLD inline
#endif

namespace bmadgpu {

constexpr real_const kPi = 3.141592653589793238462643383279;
constexpr real_const kTwoPi = 2 * kPi;
constexpr real_const kCLight = 2.99792458e8;
constexpr int kNPole = 22;

enum : int { S_ALIVE = 1, S_LOST = 2, S_NEG_X = 3, S_POS_X = 4, S_NEG_Y = 5, S_POS_Y = 6, S_LOST_PZ = 8 };
enum : int { L_UPSTREAM = 1, L_DOWNSTREAM = 2, L_INSIDE = 3 };


// Signed binomial tables of c_multi.f90:38-63: c(n,m) (c_full) and c(n,m) * n! (no_n_fact = T),
// built on the host with the reference's operation sequence and uploaded once per device.
#if defined(__CUDACC__)
__constant__ double c_cmulti[kNPole][kNPole];
__constant__ double c_cfull[kNPole][kNPole];
#define BG_CMULTI(n, m) c_cmulti[n][m]
#define BG_CFULL(n, m) c_cfull[n][m]
#else
extern double h_cmulti[kNPole][kNPole];
extern double h_cfull[kNPole][kNPole];
#define BG_CMULTI(n, m) h_cmulti[n][m]
#define BG_CFULL(n, m) h_cfull[n][m]
#endif

#if defined(BG_CR_TRANSCENDENTALS)
BG_HD double m_sin(double x) { return cr::sin(x); }
BG_HD double m_cos(double x) { return cr::cos(x); }
BG_HD double m_asin(double x) { return cr::asin(x); }
BG_HD double m_atan2(double y, double x) { return cr::atan2(y, x); }
BG_HD void m_sincos(double x, double& s, double& c) { cr::sincos(x, &s, &c); }
BG_HD void m_sinhcosh(double x, double& s, double& c) { cr::sinhcosh(x, &s, &c); }
BG_HD double m_exp(double x) { return cr::exp(x); }
BG_HD double m_tan(double x) { return cr::tan(x); }
#else
BG_HD double m_sin(double x) { return sin(x); }
BG_HD double m_cos(double x) { return cos(x); }
BG_HD double m_asin(double x) { return asin(x); }
BG_HD double m_atan2(double y, double x) { return atan2(y, x); }
BG_HD void m_sincos(double x, double& s, double& c) {
  s = sin(x);
  c = cos(x);
}
BG_HD void m_sinhcosh(double x, double& s, double& c) {
  s = sinh(x);
  c = cosh(x);
}
BG_HD double m_exp(double x) { return exp(x); }
BG_HD double m_tan(double x) { return tan(x); }
#endif

struct Particle {
  double x, px, y, py, z, pz, beta;
  int state;
  // functions of pz (and beta) the reference evaluates with the same expression in each
  // element; refreshed by refresh() whenever pz or beta change
  double dzb;               // sqrt_one(mc2**2 (2 pz + pz**2) / ((p0c (1+pz))**2 + mc2**2))  (drift dz)
  double e_factor;          // 1 / (1 + pz)                                                  (hwang edge)
  double lez_a;             // 1 - 3 (pz beta0**2)/2 + pz**2 f   or  beta - beta0           (low-energy dz)
  bool lez_series;          // series branch of low_energy_z_correction
};

BG_HD double sqrt_one(double x) {  // sim_utils/special_functions/sqrt_one.f90
  double sq = sqrt(1 + x);
  double rad = sq + 1;
  return x / rad;
}

// a / b, correctly rounded, from y = RN(1/b) shared by several quotients with the divisor b:
// q = RN(a y), r = a - b q (exact by an FMA), and RN(q + r y) = RN(a / b) (Markstein's correction
// theorem: P. Markstein, "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34 (1990) 111-119; J.-M. Muller et al., Handbook of Floating-Point
// Arithmetic, 2nd ed. (2018), sec. 4.8). The theorem needs no underflow or overflow, so quotients
// outside [2^-900, 2^900] take the plain division; a zero numerator gives q itself (the sign of the
// zero quotient is that of a y). Every caller's y is itself a rounded division 1 / b (or an exact
// power-of-two multiple of one), so each quotient is the same bits as a / b.
// Only a translation unit that defines BG_SHARED_RECIPROCAL before its includes takes the quotients
// this way (the plain tracking kernel, where it measured faster); every other one -- the batch and
// adjoint kernels, whose register-tight shapes measured slower with it, and the operation-counting
// host build -- takes a / b directly, the same bits, and leaves the shared reciprocal out (it is
// not an operation of the reference, and div_rcp then does not use it).
#if defined(BG_COUNT_OPS) || !defined(BG_SHARED_RECIPROCAL)
BG_HD double div_rcp(double a, double b, double y) {  // counted as the one division it replaces
  (void)y;
  return a / b;
}
BG_HD double shared_rcp(double b) { return b; }
BG_HD double half_rcp(double y) { return y; }
#else
BG_HD double shared_rcp(double b) { return 1 / b; }
BG_HD double half_rcp(double y) { return 0.5 * y; }  // RN(1/(2b)) from y = RN(1/b): exact scaling
BG_HD double div_rcp(double a, double b, double y) {
  const double q = a * y;
  const double aq = fabs(q);
  if (aq >= 0x1p-900 && aq <= 0x1p+900) {
    const double r = fma(-b, q, a);
    return fma(r, y, q);
  }
  if (a == 0) return q;
  return a / b;
}
#endif
constexpr real_const kRcp6 = 1.0 / 6.0;  // RN(1/6): the divisor of the Taylor terms x/6

BG_HD void refresh(Particle& p, const Globals& g) {
  double delta = p.pz;
  double rel_pc = 1 + delta;
  double pr = g.p0c * rel_pc;
  p.dzb = sqrt_one((g.mass2 * (2 * delta + delta * delta)) / (pr * pr + g.mass2));
  p.e_factor = 1 / (1 + p.pz);
  // low_energy_z_correction.f90:43-52
  double b0pz = g.beta0 * p.pz;
  p.lez_series = g.mass * (b0pz * b0pz) < g.lez_thresh;
  if (p.lez_series) p.lez_a = 1 - 3 * (p.pz * g.lez_b02) / 2 + (p.pz * p.pz) * g.lez_f;
  else p.lez_a = p.beta - g.beta0;
}

// low_energy_z_correction, bmad/low_level/low_energy_z_correction.f90:22-57
BG_HD double low_energy_z(const Particle& p, double ds, const Globals& g) {
  if (p.lez_series) return ds * p.pz * p.lez_a * g.lez_me2;
  return div_rcp(ds * p.lez_a, g.beta0, g.inv_beta0);
}

// orbit_too_large, bmad/low_level/orbit_too_large.f90:26-120
BG_HD bool orbit_too_large(Particle& p, const Globals& g) {
  if (p.x > g.max_ap) { p.state = S_POS_X; return true; }
  if (-p.x > g.max_ap) { p.state = S_NEG_X; return true; }
  if (p.y > g.max_ap) { p.state = S_POS_Y; return true; }
  if (-p.y > g.max_ap) { p.state = S_NEG_Y; return true; }
  double rel_p = 1 + p.pz;
  if (rel_p < 0) { p.state = S_LOST_PZ; return true; }
  double f = p.px * p.px + p.py * p.py - rel_p * rel_p;
  if (f > 0) {
    if (fabs(p.px) > fabs(p.py)) p.state = (p.px > 0) ? S_POS_X : S_NEG_X;
    else p.state = (p.py > 0) ? S_POS_Y : S_NEG_Y;
    return true;
  }
  return false;
}

// check_this_limit (check_aperture_limit.f90:344-356) on one coordinate
BG_HD void window_limit(Particle& p, double coord, double width2, double center, double& uf) {
  if (width2 == 0) return;
  if (coord > center - width2 && coord < center + width2) return;
  p.state = S_LOST;
  const double lo = (center - width2) - coord, hi = coord - (center + width2);
  uf = (lo < hi) ? hi : lo;  // max(lo, hi)
}

// The collimators' momentum and longitudinal windows (check_aperture_limit.f90:113-151):
// elliptical in (px, py) and (z, pz) for an ecollimator with both half widths set, else one
// check_this_limit per coordinate. Returns the unstable factor they leave.
BG_COLD double aperture_windows(Particle& p, const ApRec& a) {
  double uf = 0;
  const auto* w = a.win;
  if (a.win_kind == 1) {
    for (int k = 0; k < 2; k++) {
      const double xw = w[4 * k], x0 = w[4 * k + 1], yw = w[4 * k + 2], y0 = w[4 * k + 3];
      const double u = k == 0 ? p.px : p.z, v = k == 0 ? p.py : p.pz;
      if (xw == 0 || yw == 0) {
        window_limit(p, u, xw, x0, uf);
        window_limit(p, v, yw, y0, uf);
      } else {
        const double r = ((u - x0) / xw) * ((u - x0) / xw) + ((v - y0) / yw) * ((v - y0) / yw);
        if (r > 1) {
          p.state = S_LOST;
          uf = sqrt(r) - 1;
        }
      }
    }
  } else {
    window_limit(p, p.px, w[0], w[1], uf);
    window_limit(p, p.py, w[2], w[3], uf);
    window_limit(p, p.z, w[4], w[5], uf);
    window_limit(p, p.pz, w[6], w[7], uf);
  }
  return uf;
}

// check_aperture_limit (bmad/low_level/check_aperture_limit.f90:30-387), rectangular and
// elliptical x/y limits (offset_moves_aperture = F), after the collimator windows when present.
BG_HD void aperture(Particle& p, const ApRec& a, bool elliptical, bool windows = false) {
  double uf = 0;
  if (windows) uf = aperture_windows(p, a);
  double xp = p.x, yp = p.y;
  if (elliptical) {  // elliptical_params_setup packed: (x_width2, x0, y_width2, y0)
    const double xw = a.x1_lim, yw = a.y1_lim;
    xp = xp - a.x2_lim;
    yp = yp - a.y2_lim;
    double rx = xp / xw, ry = yp / yw;
    double r = rx * rx + ry * ry;
    if (r < 1) return;
    if (fabs(xp / xw) > fabs(yp / yw)) p.state = (xp > 0) ? S_POS_X : S_NEG_X;
    else p.state = (yp > 0) ? S_POS_Y : S_NEG_Y;
    return;
  }
  bool out = (a.x1_lim != 0 && xp < a.x1_lim) || (a.x2_lim != 0 && xp > a.x2_lim) ||
             (a.y1_lim != 0 && yp < a.y1_lim) || (a.y2_lim != 0 && yp > a.y2_lim);
  if (!out) return;
  if (a.x1_lim != 0 && xp < a.x1_lim) {
    double f = fabs((xp - a.x1_lim) / (a.x2_lim - a.x1_lim));
    if (f > uf) { p.state = S_NEG_X; uf = f; }
  }
  if (a.x2_lim != 0 && xp > a.x2_lim) {
    double f = fabs((xp - a.x2_lim) / (a.x2_lim - a.x1_lim));
    if (f > uf) { p.state = S_POS_X; uf = f; }
  }
  if (a.y1_lim != 0 && yp < a.y1_lim) {
    double f = fabs((yp - a.y1_lim) / (a.y2_lim - a.y1_lim));
    if (f > uf) { p.state = S_NEG_Y; uf = f; }
  }
  if (a.y2_lim != 0 && yp > a.y2_lim) {
    double f = fabs((yp - a.y2_lim) / (a.y2_lim - a.y1_lim));
    if (f > uf) { p.state = S_POS_Y; uf = f; }
  }
}

// track_a_drift, bmad/low_level/track_a_drift.f90:25-116 (direction = +1, with reference
// motion). sqrt(1 + (-pxy2)) equals ps_rel exactly, so sqrt_one(-pxy2) reuses it.
BG_HD void drift(Particle& p, double length) {
  if (length == 0) return;
  // quotients by 1 + pz use the particle's cached 1 / (1 + pz), those by ps_rel one reciprocal
  double rel_pc = 1 + p.pz;
  double px_rel = div_rcp(p.px, rel_pc, p.e_factor);
  double py_rel = div_rcp(p.py, rel_pc, p.e_factor);
  double pxy2 = px_rel * px_rel + py_rel * py_rel;
  if (pxy2 >= 1) { p.state = S_LOST_PZ; return; }
  double ps_rel = sqrt(1 - pxy2);
  const double inv_ps = shared_rcp(ps_rel);
  p.x = p.x + div_rcp(length * px_rel, ps_rel, inv_ps);
  p.y = p.y + div_rcp(length * py_rel, ps_rel, inv_ps);
  double dz;
  if (p.beta > 0) {
    double so = -pxy2 / (ps_rel + 1);  // sqrt_one(-pxy2)
    dz = length * (p.dzb + div_rcp(so, ps_rel, inv_ps));
  } else {
    dz = length * (1 - div_rcp(1.0, ps_rel, inv_ps));  // = RN(1 / ps_rel), the same bits as inv_ps
  }
  p.z = p.z + dz;
}

// x**m for a run-time integer m by binary powering (the lowering gfortran uses), mexp.f90
BG_HD double mexp(double x, int m) {
  if (m < 0) return 0;
  if (m == 0) return 1;
  unsigned n = (unsigned)m;
  double y = (n % 2) ? x : 1;
  while (n >>= 1) {
    x = x * x;
    if (n % 2) y = y * x;
  }
  return y;
}

// Powers x**k, k = 0..N, with exactly the roundings of mexp's binary powering: x**k is the product
// of the repeated squares x, x**2, x**4, x**8 selected by the set bits of k, taken from the lowest
// bit up, so the squares can be shared between exponents without changing any result.
template <int N>
BG_HD void mexp_table(double x, double* __restrict__ xp) {
  double sq[4];
  sq[0] = x;
#pragma unroll
  for (int i = 1; i < 4; i++) sq[i] = sq[i - 1] * sq[i - 1];
  xp[0] = 1;
#pragma unroll
  for (int k = 1; k <= N; k++) {
    double y = 0;
    bool started = false;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      if ((k >> i) & 1) {
        y = started ? y * sq[i] : sq[i];
        started = true;
      }
    }
    xp[k] = y;
  }
}

// Sum over orders n < NP of ab_multipole_kick (multipole_mod.f90:314-376), as ab_multipole_kicks
// accumulates it (:103-115). c: (b_n * scale, a_n * scale). Terms whose coefficient is exactly
// zero add an exact zero in the reference and are skipped.
template <int NP>
BG_HD void ab_kick_sum(double x, double y, const double* __restrict__ c, double& kx_tot, double& ky_tot) {
  double xp[NP], yp[NP];
  mexp_table<NP - 1>(x, xp);
  mexp_table<NP - 1>(y, yp);
  kx_tot = 0;
  ky_tot = 0;
#pragma unroll
  for (int n = 0; n < NP; n++) {
    const double b2 = c[2 * n], a2 = c[2 * n + 1];
    double kx = 0, ky = 0;
    if (!(a2 == 0 && b2 == 0)) {
#pragma unroll
      for (int m = 0; m <= n; m += 2) {
        double f = BG_CMULTI(n, m) * xp[n - m] * yp[m];
        if (b2 != 0) kx = kx + b2 * f;
        if (a2 != 0) ky = ky - a2 * f;
      }
#pragma unroll
      for (int m = 1; m <= n; m += 2) {
        double f = BG_CMULTI(n, m) * xp[n - m] * yp[m];
        if (a2 != 0) kx = kx + a2 * f;
        if (b2 != 0) ky = ky + b2 * f;
      }
    }
    kx_tot = kx_tot + kx;
    ky_tot = ky_tot + ky;
  }
}

// Any order count: the reference's loop with run-time powers.
BG_HD void ab_kick_sum_any(double x, double y, const double* __restrict__ c, int n_pole, double& kx_tot,
                           double& ky_tot) {
  kx_tot = 0;
  ky_tot = 0;
  for (int n = 0; n < n_pole; n++) {
    const double b2 = c[2 * n], a2 = c[2 * n + 1];
    double kx = 0, ky = 0;
    if (!(a2 == 0 && b2 == 0)) {
      for (int m = 0; m <= n; m += 2) {
        double f = BG_CMULTI(n, m) * mexp(x, n - m) * mexp(y, m);
        kx = kx + b2 * f;
        ky = ky - a2 * f;
      }
      for (int m = 1; m <= n; m += 2) {
        double f = BG_CMULTI(n, m) * mexp(x, n - m) * mexp(y, m);
        kx = kx + a2 * f;
        ky = ky + b2 * f;
      }
    }
    kx_tot = kx_tot + kx;
    ky_tot = ky_tot + ky;
  }
}

// The same sum when every a_n is zero and b_0 = b_1 = 0 (sextupole-like kicks): orders 2 .. NP-1
// as one branch-free block, so the independent products of all orders can be interleaved. A zero
// b_n here adds b_n f = +0 to a sum that is never -0, which is what the reference adds, so the
// bits are those of ab_kick_sum.
template <int NP>
BG_HD void ab_kick_sum_b(double x, double y, const double* __restrict__ c, double& kx_tot, double& ky_tot) {
  double xp[NP], yp[NP];
  mexp_table<NP - 1>(x, xp);
  mexp_table<NP - 1>(y, yp);
  kx_tot = 0;
  ky_tot = 0;
#pragma unroll
  for (int n = 2; n < NP; n++) {
    const double b2 = c[2 * n];
    double kx = 0, ky = 0;
#pragma unroll
    for (int m = 0; m <= n; m += 2) {
      const double f = BG_CMULTI(n, m) * xp[n - m] * yp[m];
      kx = kx + b2 * f;
    }
#pragma unroll
    for (int m = 1; m <= n; m += 2) {
      const double f = BG_CMULTI(n, m) * xp[n - m] * yp[m];
      ky = ky + b2 * f;
    }
    kx_tot = kx_tot + kx;
    ky_tot = ky_tot + ky;
  }
}

BG_HD void ab_kick_dispatch_b(double x, double y, const double* __restrict__ c, int n_pole, double& kx, double& ky) {
  switch (n_pole) {
    case 3: ab_kick_sum_b<3>(x, y, c, kx, ky); break;
    case 4: ab_kick_sum_b<4>(x, y, c, kx, ky); break;
    case 5: ab_kick_sum_b<5>(x, y, c, kx, ky); break;
    case 6: ab_kick_sum_b<6>(x, y, c, kx, ky); break;
    case 7: ab_kick_sum_b<7>(x, y, c, kx, ky); break;
    case 8: ab_kick_sum_b<8>(x, y, c, kx, ky); break;
    case 9: ab_kick_sum_b<9>(x, y, c, kx, ky); break;
    case 10: ab_kick_sum_b<10>(x, y, c, kx, ky); break;
    case 11: ab_kick_sum_b<11>(x, y, c, kx, ky); break;
    default: ab_kick_sum_any(x, y, c, n_pole, kx, ky); break;
  }
}

BG_HD void ab_kick_dispatch(double x, double y, const double* __restrict__ c, int n_pole, double& kx, double& ky) {
  switch (n_pole) {
    case 1: ab_kick_sum<1>(x, y, c, kx, ky); break;
    case 2: ab_kick_sum<2>(x, y, c, kx, ky); break;
    case 3: ab_kick_sum<3>(x, y, c, kx, ky); break;
    case 4: ab_kick_sum<4>(x, y, c, kx, ky); break;
    case 5: ab_kick_sum<5>(x, y, c, kx, ky); break;
    case 6: ab_kick_sum<6>(x, y, c, kx, ky); break;
    case 7: ab_kick_sum<7>(x, y, c, kx, ky); break;
    case 8: ab_kick_sum<8>(x, y, c, kx, ky); break;
    case 9: ab_kick_sum<9>(x, y, c, kx, ky); break;
    case 10: ab_kick_sum<10>(x, y, c, kx, ky); break;
    case 11: ab_kick_sum<11>(x, y, c, kx, ky); break;
    default: ab_kick_sum_any(x, y, c, n_pole, kx, ky); break;
  }
}

// ab_multipole_kicks (multipole_mod.f90:82-121), magnetic, coefficients pre-scaled; b_from2: the
// element's kicks carry F_KICK_B_FROM2.
BG_HD void ab_kicks(Particle& p, const double* __restrict__ c, int n_pole, bool b_from2 = false) {
  double kx_tot, ky_tot;
  if (b_from2)
    ab_kick_dispatch_b(p.x, p.y, c, n_pole, kx_tot, ky_tot);
  else
    ab_kick_dispatch(p.x, p.y, c, n_pole, kx_tot, ky_tot);
  p.px = p.px + kx_tot;
  p.py = p.py + ky_tot;
}

// Field of the bend multipoles (ab_multipole_kick with ele_orientation = 0, unscaled) as
// track_a_bend's apply_multipole_kicks sums it (track_a_bend.f90:366-379).
BG_HD void ab_field(const Particle& p, const double* __restrict__ c, int n_pole, double f_p0c, double& B1,
                    double& B2) {
  B1 = 0;
  B2 = 0;
  const double x = p.x, y = p.y;
  for (int n = 0; n < n_pole; n++) {
    const double b = c[2 * n], a = c[2 * n + 1];
    if (a == 0 && b == 0) continue;
    double kx = 0, ky = 0;
    for (int m = 0; m <= n; m += 2) {
      double f = BG_CMULTI(n, m) * mexp(x, n - m) * mexp(y, m);
      kx = kx + b * f;
      ky = ky - a * f;
    }
    for (int m = 1; m <= n; m += 2) {
      double f = BG_CMULTI(n, m) * mexp(x, n - m) * mexp(y, m);
      kx = kx + a * f;
      ky = ky + b * f;
    }
    B1 = B1 + f_p0c * ky;
    B2 = B2 - f_p0c * kx;
  }
}

// multipole_kick (multipole_mod.f90:203-286), magnetic, n >= 1, tilt given by cos/sin (t_zero
// when the tilt is exactly zero).
BG_HD void thin_kick(Particle& p, double knl, int n, bool t_zero, double cos_ang, double sin_ang) {
  double x, y;
  if (t_zero) {
    x = p.x;
    y = p.y;
  } else {
    x = p.x * cos_ang + p.y * sin_ang;
    y = -p.x * sin_ang + p.y * cos_ang;
  }
  double x_terms[kNPole], y_terms[kNPole];
  x_terms[n] = 1.0;
  y_terms[0] = 1.0;
  for (int m = 1; m <= n; m++) {
    x_terms[n - m] = x_terms[n - m + 1] * x;
    y_terms[m] = y_terms[m - 1] * y;
  }
  double x_value = 0, y_value = 0;
  for (int m = 0; m <= n; m += 2) x_value = x_value + BG_CFULL(n, m) * x_terms[m] * y_terms[m];
  for (int m = 1; m <= n; m += 2) y_value = y_value + BG_CFULL(n, m) * x_terms[m] * y_terms[m];
  double x_vel = 1.0 * knl * x_value;
  double y_vel = 1.0 * knl * y_value;
  if (t_zero) {
    p.px = p.px + x_vel;
    p.py = p.py + y_vel;
  } else {
    p.px = p.px + x_vel * cos_ang - y_vel * sin_ang;
    p.py = p.py + x_vel * sin_ang + y_vel * cos_ang;
  }
}

// tilt_coords, bmad/code/tilt_coords.f90:18-53 (cos/sin precomputed; Fortran matmul order)
BG_HD void tilt(Particle& p, double c, double s) {
  double x = p.x, y = p.y, px = p.px, py = p.py;
  p.x = (0 + c * x) + s * y;
  p.y = (0 + -s * x) + c * y;
  p.px = (0 + c * px) + s * py;
  p.py = (0 + -s * px) + c * py;
}

// track_a_drift without the reference motion (include_ref_motion = .false.,
// track_a_drift.f90:25-116): the drift of offset_particle to the element's nominal edge.
BG_HD void drift_noref(Particle& p, double length) {
  double rel_pc = 1 + p.pz;
  double px_rel = div_rcp(p.px, rel_pc, p.e_factor);
  double py_rel = div_rcp(p.py, rel_pc, p.e_factor);
  double pxy2 = px_rel * px_rel + py_rel * py_rel;
  if (pxy2 >= 1) { p.state = S_LOST_PZ; return; }
  double ps_rel = sqrt(1 - pxy2);
  const double inv_ps = shared_rcp(ps_rel);
  p.x = p.x + div_rcp(length * px_rel, ps_rel, inv_ps);
  p.y = p.y + div_rcp(length * py_rel, ps_rel, inv_ps);
  p.z = p.z + 1 * div_rcp(-length, ps_rel, inv_ps);
}

// Fortran matmul(w, r) for a 3x3 w (row-major here), summed in the order of the inlined loop.
BG_HD void matvec3(const double* __restrict__ w, const double r[3], double out[3]) {
  for (int i = 0; i < 3; i++) out[i] = ((0 + w[3 * i] * r[0]) + w[3 * i + 1] * r[1]) + w[3 * i + 2] * r[2];
}

// offset_particle set/unset of straight elements with pitches or z_offset (offset_particle.f90:
// 239-258, 279-282 set; 437-458, 477-480 unset): the offset position rotated by W^-1 (set) or W
// (unset), the momentum by the same rotation, then the drift to the nominal edge; the tilt last
// (set) or first (unset). m: the 27-double misalign block (table.h).
BG_COLD void offset_set_pitched(Particle& p, const double* __restrict__ m, bool has_tilt) {
  const double L_half = m[5], ds_center = m[6];
  const double r[3] = {p.x - m[0], p.y - m[1], 0.0 - (m[4] + 1 * ds_center)};
  double q[3];
  matvec3(m + 9, r, q);
  q[2] = q[2] + L_half;
  const double s_body = q[2];
  const double rel_p = 1 + p.pz;
  const double pz2 = rel_p * rel_p - p.px * p.px - p.py * p.py;
  if (pz2 <= 0) {
    p.state = S_LOST_PZ;
  } else {
    const double v[3] = {p.px, p.py, 1 * sqrt(pz2)};
    double pv[3];
    matvec3(m + 9, v, pv);
    p.px = pv[0];
    p.py = pv[1];
    p.x = q[0];
    p.y = q[1];
  }
  const double ds = (1 - 1) * L_half - s_body;
  if (fabs(ds) > 1e-14 && p.state == S_ALIVE) drift_noref(p, ds);
  if (has_tilt) tilt(p, m[2], m[3]);
}
BG_COLD void offset_unset_pitched(Particle& p, const double* __restrict__ m, bool has_tilt) {
  if (has_tilt) tilt(p, m[2], -m[3]);
  const double L_half = m[5];
  double r[3] = {p.x, p.y, 0.0};
  r[2] = r[2] - m[7];
  double q[3];
  matvec3(m + 18, r, q);
  q[0] = q[0] + m[0];
  q[1] = q[1] + m[1];
  q[2] = q[2] + (m[4] + L_half);
  const double s_lab = q[2];
  const double rel_p = 1 + p.pz;
  const double pz2 = rel_p * rel_p - p.px * p.px - p.py * p.py;
  if (pz2 <= 0) {
    p.state = S_LOST_PZ;
  } else {
    const double v[3] = {p.px, p.py, 1 * sqrt(pz2)};
    double pv[3];
    matvec3(m + 18, v, pv);
    p.px = pv[0];
    p.py = pv[1];
    p.x = q[0];
    p.y = q[1];
  }
  const double ds = m[8] - s_lab;
  if (fabs(ds) > 1e-14 && p.state == S_ALIVE) drift_noref(p, ds);
}

// offset_particle set/unset for straight elements with x/y offsets and tilt, no pitches or
// z_offset (offset_particle.f90:201-330, 374-459): the transforms reduce to exact shifts, the
// pz-loss test and tilt_coords; no drift to the edge is needed (s_body = s_target). With
// pitched, the general form above.
BG_HD void offset_set(Particle& p, const double* __restrict__ m, bool has_tilt, bool pitched = false) {
  if (pitched) {
    offset_set_pitched(p, m, has_tilt);
    return;
  }
  if (m[0] != 0 || m[1] != 0) {
    p.x = p.x - m[0];
    p.y = p.y - m[1];
    double rel_p = 1 + p.pz;
    if (rel_p * rel_p - p.px * p.px - p.py * p.py <= 0) p.state = S_LOST_PZ;
  }
  if (has_tilt) tilt(p, m[2], m[3]);
}
BG_HD void offset_unset(Particle& p, const double* __restrict__ m, bool has_tilt, bool pitched = false) {
  if (pitched) {
    offset_unset_pitched(p, m, has_tilt);
    return;
  }
  if (has_tilt) tilt(p, m[2], -m[3]);
  if (m[0] != 0 || m[1] != 0) {
    double rel_p = 1 + p.pz;
    if (rel_p * rel_p - p.px * p.px - p.py * p.py <= 0) p.state = S_LOST_PZ;
    p.x = p.x + m[0];
    p.y = p.y + m[1];
  }
}

// quad_mat2_calc, bmad/low_level/quad_mat2_calc.f90:22-61 (mat2 and z_coef)
// ef = RN(1 / rel_p), shared by the quotients by rel_p and 2 rel_p.
// The part of quad_mat2_calc after cx, sx (quad_mat2_calc.f90:49-61).
BG_HD void quad_mat2_tail(double k1, double length, double rel_p, double ef, double cx, double sx, double& m11,
                          double& m12, double& m21, double& m22, double& z0, double& z1, double& z2) {
  m11 = cx;
  m12 = div_rcp(sx, rel_p, ef);
  m21 = k1 * sx * rel_p;
  m22 = cx;
  z0 = k1 * (-cx * sx + length) / 4;
  z1 = div_rcp(-k1 * (sx * sx), 2 * rel_p, half_rcp(ef));
  z2 = -(cx * sx + length) / (4 * (rel_p * rel_p));
}

BG_HD void quad_mat2(double k1, double length, double rel_p, double ef, double& m11, double& m12, double& m21,
                     double& m22, double& z0, double& z1, double& z2) {
  double sqrt_k = sqrt(fabs(k1));
  double sk_l = sqrt_k * length;
  double cx, sx;
  if (fabs(sk_l) < 1e-10) {
    double k_l2 = k1 * (length * length);
    cx = 1 + k_l2 / 2;
    sx = (1 + div_rcp(k_l2, 6, kRcp6)) * length;
  } else if (k1 < 0) {
    double s;
    m_sincos(sk_l, s, cx);
    sx = s / sqrt_k;
  } else {
    double s;
    m_sinhcosh(sk_l, s, cx);
    sx = s / sqrt_k;
  }
  quad_mat2_tail(k1, length, rel_p, ef, cx, sx, m11, m12, m21, m22, z0, z1, z2);
}

// Both planes of a quadrupole step, x with -k1 and y with k1, as two quad_mat2 calls give them.
// One plane takes cos/sin and the other cosh/sinh of the same sqrt(|k1|) L; evaluating the four
// in one block, with the planes picked by the reference's sign tests, lets the two independent
// chains interleave. The calls and their arguments are those of quad_mat2, so are the bits.
BG_HD void quad_mat2_xy(double k1, double length, double rel_p, double ef, double* mx, double* my) {
  const double sqrt_k = sqrt(fabs(k1));
  const double sk_l = sqrt_k * length;
  double cxx, sxx, cxy, sxy;
  if (fabs(sk_l) < 1e-10) {
    const double kl2x = -k1 * (length * length), kl2y = k1 * (length * length);
    cxx = 1 + kl2x / 2;
    sxx = (1 + div_rcp(kl2x, 6, kRcp6)) * length;
    cxy = 1 + kl2y / 2;
    sxy = (1 + div_rcp(kl2y, 6, kRcp6)) * length;
  } else {
    double c_t, s_t, c_h, s_h;
    m_sincos(sk_l, s_t, c_t);
    m_sinhcosh(sk_l, s_h, c_h);
    s_t = s_t / sqrt_k;
    s_h = s_h / sqrt_k;
    const bool x_trig = -k1 < 0, y_trig = k1 < 0;
    cxx = x_trig ? c_t : c_h;
    sxx = x_trig ? s_t : s_h;
    cxy = y_trig ? c_t : c_h;
    sxy = y_trig ? s_t : s_h;
  }
  quad_mat2_tail(-k1, length, rel_p, ef, cxx, sxx, mx[0], mx[1], mx[2], mx[3], mx[4], mx[5], mx[6]);
  quad_mat2_tail(k1, length, rel_p, ef, cxy, sxy, my[0], my[1], my[2], my[3], my[4], my[5], my[6]);
}

// One body step of track_a_quadrupole (track_a_quadrupole.f90:95-120); b1 and length are the
// element's (charge_dir = 1).
BG_HD void quad_step(Particle& p, double b1, double length, double step_len, const Globals& G) {
  double rel_p = 1 + p.pz;
  double k1 = b1 / (length * rel_p);
  double mx[7], my[7];
  quad_mat2_xy(k1, step_len, rel_p, p.e_factor, mx, my);
  const double ax = mx[0], bx = mx[1], cx_ = mx[2], dx = mx[3], zx0 = mx[4], zx1 = mx[5], zx2 = mx[6];
  const double ay = my[0], by = my[1], cy = my[2], dy = my[3], zy0 = my[4], zy1 = my[5], zy2 = my[6];
  double x = p.x, px = p.px, y = p.y, py = p.py;
  p.z = p.z + (zx0 * (x * x) + zx1 * x * px + zx2 * (px * px) + zy0 * (y * y) + zy1 * y * py + zy2 * (py * py));
  p.x = (0 + ax * x) + bx * px;
  p.px = (0 + cx_ * x) + dx * px;
  p.y = (0 + ay * y) + by * py;
  p.py = (0 + cy * y) + dy * py;
  p.z = p.z + low_energy_z(p, step_len, G);
}

// hwang_bend_edge_kick, bmad/modules/fringe_mod.f90:241-419 (time_dir = +1).
// e: [gt, gt2, gs2, k1_tane, fg_factor, g_tot, gt*g_tot*(1 + 2 tan_e**2)]
BG_HD void hwang_edge(Particle& p, const double* __restrict__ e, bool entering) {
  double gt = e[0], gt2 = e[1], gs2 = e[2], k1t = e[3], fg = e[4], gtot = e[5], cdpx = e[6];
  double ef = p.e_factor;
  double v1 = p.x, v2 = p.px, v3 = p.y, v4 = p.py;
  double v11 = v1 * v1, v33 = v3 * v3;
  double dx, dpx, dy, dpy, dz;
  if (entering) {
    dx = (-gt2 * v11 + gs2 * v33) * ef / 2;
    dpx = (cdpx * v33 / 2 + gt2 * (v1 * v2 - v3 * v4) + k1t * (v11 - v33)) * ef;
    dy = gt2 * v1 * v3 * ef;
    dpy = (fg * v3 - gt2 * v1 * v4 - (gtot + gt2) * v2 * v3 - 2 * k1t * v1 * v3) * ef;
    dz = (ef * ef) * 0.5 *
         (v33 * fg + div_rcp((v11 * v1) * (4.0 * k1t - gt * gt2), 6.0, kRcp6) + 0.5 * v1 * v33 * (-4.0 * k1t + gt * gs2) +
          (v11 * v2 - 2.0 * v1 * v3 * v4) * gt2 - v2 * v33 * gs2);
  } else {
    dx = (gt2 * v11 - gs2 * v33) * ef / 2;
    dpx = (gt2 * (v3 * v4 - v1 * v2) + k1t * (v11 - v33) - gt * gt2 * (v11 + v33) / 2) * ef;
    dy = -gt2 * v1 * v3 * ef;
    dpy = (fg * v3 + gt2 * v1 * v4 + (gtot + gt2) * v2 * v3 + (gt * gs2 - 2 * k1t) * v1 * v3) * ef;
    dz = (ef * ef) * 0.5 *
         (v33 * fg + div_rcp((v11 * v1) * (4.0 * k1t - gt * gt2), 6.0, kRcp6) + 0.5 * v1 * v33 * (-4.0 * k1t + gt * gs2) -
          (v11 * v2 - 2.0 * v1 * v3 * v4) * gt2 + v2 * v33 * gs2);
  }
  p.x = v1 + 1.0 * dx;
  p.px = v2 + 1.0 * (dpx + gt * v1);
  p.y = v3 + 1.0 * dy;
  p.py = v4 + 1.0 * (dpy - gt * v3);
  p.z = p.z + 1.0 * dz;
}

// sbend_body_with_k1_map, track_a_bend.f90:500-659 (ending coordinates only).
// b: bend parameter block (table.h); k1 = b1 / L in b[10], the step length in b[0].
BG_HD void bend_k1_step(Particle& p, const double* __restrict__ b) {
  double length = b[0], g = b[1], g_tot = b[2], k1 = b[10];
  double rel_p = 1 + p.pz, rel_p2 = rel_p * rel_p;
  double k_x = k1 + g * g_tot;
  double x_c = (g * rel_p - g_tot) / k_x;
  double om_x = sqrt(fabs(k_x) / rel_p), om_y = sqrt(fabs(k1) / rel_p);
  double tau_x = (k_x >= 0) ? -1.0 : 1.0, tau_y = (k1 >= 0) ? 1.0 : -1.0;
  double s_x, c_x, z2, s_y, c_y, arg = om_x * length;
  if (arg < 1e-6) {
    s_x = (1 + tau_x * (arg * arg) / 6) * length;
    c_x = 1 + tau_x * (arg * arg) / 2;
    z2 = g * (length * length) / (2 * rel_p);
  } else if (k_x > 0) {
    m_sincos(arg, s_x, c_x);
    s_x = s_x / om_x;
    z2 = tau_x * g * (1 - c_x) / (rel_p * (om_x * om_x));
  } else {
    m_sinhcosh(arg, s_x, c_x);
    s_x = s_x / om_x;
    z2 = tau_x * g * (1 - c_x) / (rel_p * (om_x * om_x));
  }
  arg = om_y * length;
  if (arg < 1e-6) {
    s_y = (1 + tau_y * (arg * arg) / 6) * length;
    c_y = 1 + tau_y * (arg * arg) / 2;
  } else if (k1 < 0) {
    m_sincos(om_y * length, s_y, c_y);
    s_y = s_y / om_y;
  } else {
    m_sinhcosh(om_y * length, s_y, c_y);
    s_y = s_y / om_y;
  }
  double r1 = p.x - x_c, r2 = p.px, r3 = p.y, r4 = p.py, r5 = p.z;
  double z0 = -g * x_c * length, z1 = -g * s_x;
  double ox2 = om_x * om_x, oy2 = om_y * om_y;
  double z11 = tau_x * ox2 * (length - c_x * s_x) / 4, z12 = -tau_x * ox2 * (s_x * s_x) / (2 * rel_p);
  double z22 = -(length + c_x * s_x) / (4 * rel_p2);
  double z33 = tau_y * oy2 * (length - c_y * s_y) / 4, z34 = -tau_y * oy2 * (s_y * s_y) / (2 * rel_p);
  double z44 = -(length + c_y * s_y) / (4 * rel_p2);
  p.x = c_x * r1 + s_x * r2 / rel_p + x_c;
  p.px = tau_x * ox2 * rel_p * s_x * r1 + c_x * r2;
  p.y = c_y * r3 + s_y * r4 / rel_p;
  p.py = tau_y * oy2 * rel_p * s_y * r3 + c_y * r4;
  p.z = r5 + 1.0 * 1.0 * z0 + z1 * r1 + z2 * r2 + z11 * (r1 * r1) + z12 * r1 * r2 + z22 * (r2 * r2) +
        z33 * (r3 * r3) + z34 * r3 * r4 + z44 * (r4 * r4);
}

// Exact sbend body step, track_a_bend.f90:121-209. Returns false if the particle was lost.
BG_HD bool bend_exact_step(Particle& p, const double* __restrict__ b, const Globals& G) {
  double step_len = b[0], g = b[1], g_tot = b[2], dg = b[3], angle = b[4];
  double cos_a = b[5], sin_a = b[6], sinc_a = b[7], cosc_a = b[8], gl2_sincc = b[9];
  double x = p.x, px = p.px, y = p.y, py = p.py, z = p.z, pz = p.pz;
  double rel_p = 1 + pz;
  double rel_p2 = rel_p * rel_p;
  if (dg == 0 && fabs(x * g) < 1e-9 && fabs(px) < 1e-9 && fabs(py) < 1e-9 && fabs(pz) < 1e-9) {
    // semi-linear map near the zero orbit, track_a_bend.f90:136-159
    double ll = step_len;
    double rpp = rel_p * G.p0c;
    double gam2 = G.mass2 / (rpp * rpp + G.mass2);
    double m56 = ll * (gam2 - gl2_sincc);
    p.x = cos_a * x + ll * sinc_a * px + g * (ll * ll) * cosc_a * pz;
    p.px = -g * sin_a * x + cos_a * px + g * ll * sinc_a * pz;
    p.y = y + ll * py;
    p.z = -g * ll * sinc_a * x - g * (ll * ll) * cosc_a * px + z + m56 * pz;
    return true;
  }
  double pt = sqrt(rel_p2 - py * py);
  if (fabs(px) > pt) { p.state = S_LOST_PZ; return false; }
  const double inv_pt = shared_rcp(pt);  // shared by the four quotients by pt
  double g_p = div_rcp(g_tot, pt, inv_pt);
  double phi_1 = m_asin(div_rcp(px, pt, inv_pt));
  double cos_plus, sin_plus;
  m_sincos(angle + phi_1, sin_plus, cos_plus);
  double gx1 = 1 + g * x;
  double ls = gx1 * step_len * sinc_a;
  double alpha = 2 * gx1 * sin_plus * step_len * sinc_a - g_p * (ls * ls);
  double r = cos_plus * cos_plus + g_p * alpha;
  if (r < 0 || (fabs(g_p) < 1e-5 && fabs(cos_plus) < 1e-5)) {
    p.state = S_LOST;
    p.x = 2 * G.max_ap;
    return false;
  }
  double rad = sqrt(r);
  double xi;
  if (cos_plus > 0) {
    double denom = rad + cos_plus;
    xi = alpha / denom;
  } else {
    double denom = rad - cos_plus;
    xi = denom / g_p;
  }
  p.x = x * cos_a - (step_len * step_len) * g * cosc_a + xi;
  if (fabs(p.x) > G.max_ap) { p.state = S_LOST; return false; }
  double L_u = xi;
  double L_v = -1 * (step_len * sinc_a + x * sin_a);
  double L_c = sqrt(L_v * L_v + L_u * L_u);
  double angle_p = 2 * (angle + phi_1 - 1 * m_atan2(L_u, -L_v));
  double hp = angle_p / 2;
  double L_p = 1 * L_c / ((fabs(hp) < 1e-8) ? 1.0 : m_sin(hp) / hp);
  p.px = pt * m_sin(phi_1 + angle - angle_p);
  p.y = y + div_rcp(py * L_p, pt, inv_pt);
  p.z = z + div_rcp(p.beta * step_len, G.beta0, G.inv_beta0) - div_rcp(rel_p * L_p, pt, inv_pt);
  return true;
}

// apply_energy_kick, bmad/low_level/apply_energy_kick.f90:23-74
BG_HD void energy_kick(Particle& p, double dE, const Globals& G) {
  double mc2 = G.mass;
  double p0c = G.p0c;
  double pc = (1 + p.pz) * p0c;
  double beta_old = p.beta;
  double E_old = pc / p.beta;
  double E_new = E_old + dE;
  if (E_new < mc2) {
    p.pz = -1;
    p.beta = 0;
    p.state = S_LOST_PZ;
    return;
  }
  p.pz = p.pz + (1 + p.pz) * sqrt_one((2 * E_old * dE + dE * dE) / (pc * pc));
  double pc_new = p0c * (1 + p.pz);
  double beta_new = pc_new / E_new;
  p.z = p.z * beta_new / beta_old;
  p.beta = beta_new;
}

// ---- electric multipoles (bmad_standard field, exact_multipoles = off) -----------------------
// e: the electric block (table.h): [n_elec, scales, edge modes, at_sign charges, mass/p0c] then
// (b_n, a_n), n < n_elec.

// ab_multipole_kicks with pole_type = electric (multipole_mod.f90:82-141 with
// ab_multipole_kick :314-376): kick strengths charge / (beta p0c) times (a_n, -b_n) times scale,
// summed over the orders, then the energy change that goes with the transverse kick (the
// particle keeps its total energy in the static field), beta and z rescaled.
BG_COLD void elec_kicks(Particle& p, const double* __restrict__ e, double scale, const Globals& G) {
  const int n_pole = (int)e[0];
  const double* c = e + EL_FIXED;
  const double f = G.charge / (p.beta * G.p0c);
  const double x = p.x, y = p.y;
  double kx_tot = 0, ky_tot = 0;
  for (int n = 0; n < n_pole; n++) {
    const double b = c[2 * n], a = c[2 * n + 1];
    double kx = 0, ky = 0;
    if (!(a == 0 && b == 0)) {
      double a2 = a * f, b2 = -b * f;
      a2 = scale * a2;
      b2 = scale * b2;
      for (int m = 0; m <= n; m += 2) {
        const double t = BG_CMULTI(n, m) * mexp(x, n - m) * mexp(y, m);
        kx = kx + b2 * t;
        ky = ky - a2 * t;
      }
      for (int m = 1; m <= n; m += 2) {
        const double t = BG_CMULTI(n, m) * mexp(x, n - m) * mexp(y, m);
        kx = kx + a2 * t;
        ky = ky + b2 * t;
      }
    }
    kx_tot = kx_tot + kx;
    ky_tot = ky_tot + ky;
  }
  const double px0 = p.px, py0 = p.py, pz0 = p.pz, z0 = p.z, beta0 = p.beta;
  p.px = p.px + kx_tot;
  p.py = p.py + ky_tot;
  const double rp0 = 1 + pz0;
  const double alpha = (kx_tot * (2 * px0 + kx_tot) + ky_tot * (2 * py0 + ky_tot)) / (rp0 * rp0);
  if (alpha < -1) {
    p.state = S_LOST_PZ;
    return;
  }
  const double dpz = (1 + pz0) * sqrt_one(alpha);
  p.pz = pz0 + dpz;
  const double rp1 = 1 + p.pz;
  const double mp = e[7];
  p.beta = (1 + p.pz) / sqrt(rp1 * rp1 + mp * mp);
  p.z = z0 * p.beta / beta0;
  refresh(p, G);
}

// electric_longitudinal_fringe (apply_element_edge_kick.f90:283-329, bmad_standard field, non-exact
// multipoles): the energy kick of the scalar potential phi = -Re sum (b_n - i a_n)(x + i y)^(n+1)/(n+1)
// at the edge, ff = at_sign * charge.
BG_COLD void elec_fringe(Particle& p, const double* __restrict__ e, double ff, const Globals& G) {
  const int n_pole = (int)e[0];
  const double* c = e + EL_FIXED;
  const double cr = p.x, ci = p.y;
  double xr = 1, xi = 0, phi = 0;
  for (int i = 0; i < n_pole; i++) {
    const double nr = xr * cr - xi * ci, ni = xr * ci + xi * cr;
    xr = nr;
    xi = ni;
    const double b = c[2 * i], a = c[2 * i + 1];
    if (a == 0 && b == 0) continue;
    const double ar = b, ai = -a;
    const double re_cur = ar * xr - ai * xi;
    phi = phi - re_cur / (i + 1);
  }
  energy_kick(p, -ff * phi, G);
  refresh(p, G);
}

// ---- higher-order edge fringes (fringe_mod.f90) ----------------------------------------------
// x: the extra block (table.h).

// hard_multipole_edge_kick (fringe_mod.f90:692-865, no matrix): the hard-edge fringe of the
// order-n (1 quadrupole, 2 sextupole) component, strength x[9], as a transverse map with the
// Jacobian's determinant correcting the momenta. Complex arithmetic written out.
BG_COLD void hard_edge(Particle& p, const double* __restrict__ xb, bool entering) {
  const int n_max = (int)xb[8];
  const double x = p.x, y = p.y;
  double pr = x, pi = y;          // poly
  double fx = 0, dfx_dx = 0, dfx_dy = 0, fy = 0, dfy_dx = 0, dfy_dy = 0;
  const double rel_p = 1 + p.pz;
  for (int n = 1; n <= n_max; n++) {
    const double n1r = pr, n1i = pi;                       // poly_n1
    const double qr = pr * x - pi * y, qi = pr * y + pi * x;  // poly * xy
    pr = qr;
    pi = qi;
    if (n != n_max) continue;     // only the order of the element's own field is non-zero
    const double dxr = (n + 1) * n1r, dxi = (n + 1) * n1i;  // dpoly_dx
    const double dyr = -dxi, dyi = dxr;                      // i dpoly_dx
    const double div = 4 * (n + 2) * rel_p;
    double cr = 1.0 * xb[9], ci = 1.0 * 0.0;
    cr = cr / div;
    ci = ci / div;
    if (entering) {
      cr = -cr;
      ci = -ci;
    }
    const double cn = (double)(n + 3) / (n + 1);
    // f = Re(cab * poly * xny) and its x, y derivatives, xny = x - i cn y
    double xr = x, xi = -cn * y;
    double ar = cr * pr - ci * pi, ai = cr * pi + ci * pr;   // cab * poly
    fx = fx + (ar * xr - ai * xi);
    double tr = (dxr * xr - dxi * xi) + pr, ti = (dxr * xi + dxi * xr) + pi;
    dfx_dx = dfx_dx + (cr * tr - ci * ti);
    {
      const double ur = dyr * xr - dyi * xi, ui = dyr * xi + dyi * xr;
      const double wr = pr * 0.0 - pi * -cn, wi = pr * -cn + pi * 0.0;  // poly * dxny_dy
      tr = ur + wr;
      ti = ui + wi;
      dfx_dy = dfx_dy + (cr * tr - ci * ti);
    }
    xr = y;
    xi = cn * x;                  // xny = y + i cn x
    fy = fy + (ar * xr - ai * xi);
    {
      const double ur = dxr * xr - dxi * xi, ui = dxr * xi + dxi * xr;
      const double wr = pr * 0.0 - pi * cn, wi = pr * cn + pi * 0.0;    // poly * dxny_dx
      tr = ur + wr;
      ti = ui + wi;
      dfy_dx = dfy_dx + (cr * tr - ci * ti);
    }
    tr = (dyr * xr - dyi * xi) + pr;
    ti = (dyr * xi + dyi * xr) + pi;
    dfy_dy = dfy_dy + (cr * tr - ci * ti);
  }
  const double px = p.px, py = p.py;
  const double denom = (1 - dfx_dx) * (1 - dfy_dy) - dfx_dy * dfy_dx;
  p.x = p.x - fx;
  p.px = px + ((1.0 - dfy_dy - denom) * px + dfy_dx * py) / denom;
  p.y = p.y - fy;
  p.py = py + (dfx_dy * px + (1.0 - dfx_dx - denom) * py) / denom;
  p.z = p.z + (p.px * fx + p.py * fy) / rel_p;
}

// soft_quadrupole_edge_kick (fringe_mod.f90:556-661, no matrix): the soft-edge quadrupole fringe
// with the integrals fq1, fq2.
BG_COLD void soft_quad_edge(Particle& p, const double* __restrict__ xb, bool entering) {
  const double rel_p = 1 + p.pz;
  const double k1_rel = 1.0 * xb[10] / rel_p;
  double f1 = k1_rel * xb[11];
  const double f2 = k1_rel * xb[12];
  if (f1 == 0 && f2 == 0) return;
  if (!entering) f1 = -f1;
  const double ef1 = m_exp(f1);
  const double v0 = p.x, v1 = p.px, v2 = p.y, v3 = p.py;
  const double vx = v1 / rel_p, vy = v3 / rel_p;
  p.z = p.z - (f1 * v0 + f2 * (1 + f1 / 2) * vx / ef1) * vx + (f1 * v2 + f2 * (1 - f1 / 2) * vy * ef1) * vy;
  p.x = v0 * ef1 + vx * f2;
  p.px = v1 / ef1;
  p.y = v2 / ef1 - vy * f2;
  p.py = v3 * ef1;
}

// bmad_rot_xz (fringe_mod.f90:1691-1771) and bmad_wedger (:1563-1690), no matrix: the rotation of
// the reference frame by the edge angle, in a field g_tot for the wedger.
BG_HD bool rot_xz(double a, double* __restrict__ v) {
  const double x = v[0], px = v[1], py = v[3];
  const double pp = 1 + v[5];
  double ps = pp * pp - px * px - py * py;
  if (ps <= 0) return false;
  ps = sqrt(ps);
  const double ca = m_cos(a), sa = m_sin(a);
  const double den = ps * ca - px * sa;
  const double L = x * sa / den;
  v[0] = x * ps / den;
  v[1] = px * ca + ps * sa;
  v[2] = v[2] + py * L;
  v[4] = v[4] - pp * L;
  return true;
}
BG_HD bool wedger(double a, double g_tot, double* __restrict__ v) {
  const double b1 = g_tot;
  if (b1 == 0) return rot_xz(a, v);
  const double x = v[0], px = v[1], py = v[3];
  const double pp = 1 + v[5];
  double ps = pp * pp - px * px - py * py;
  if (ps <= 0) return false;
  ps = sqrt(ps);
  double pt = pp * pp - py * py;
  if (pt < 1e-10) return false;
  pt = sqrt(pt);
  const double ca = m_cos(a), sa = m_sin(a), s2a = m_sin(2.0 * a), s2 = sa * sa;
  const double pxn = px * ca + (ps - b1 * x) * sa;
  double psn = pt * pt - pxn * pxn;
  if (psn < 1e-10) return false;
  psn = sqrt(psn);
  const double den = psn + ps * ca - px * sa;
  const double num = x * px * s2a + s2 * (2 * x * ps - b1 * (x * x));
  const double L = (a + m_asin(px / pt) - m_asin(pxn / pt)) / b1;
  v[0] = x * ca + num / den;
  v[1] = pxn;
  v[2] = v[2] + py * L;
  v[4] = v[4] - pp * L;
  return true;
}

// bmad_fringe_dipoler (fringe_mod.f90:1772-1933, no matrix): the hard-edge dipole fringe with the
// fringe integral fint hgap.
BG_HD bool fringe_dipoler(double* __restrict__ v, double g_tot, double beta0, double fint, double hgap,
                          bool entering) {
  const double b = entering ? g_tot : -g_tot;
  const double x = v[0], px = v[1], y = v[2], py = v[3], z = v[4];
  const double pp = 1 + v[5];
  double ps = pp * pp - px * px - py * py;
  if (ps <= 0) return false;
  ps = sqrt(ps);
  const double ee = sqrt(pp * pp + 1 / (beta0 * beta0) - 1);
  const double beta = pp / ee;
  const double xp = px / ps, yp = py / ps;
  const double kap = b * fint * hgap;
  const double fac2 = 1 + yp * yp;
  const double d11 = (1 + xp * xp) / ps, d21 = xp * yp / ps, d31 = -xp;
  const double d12 = xp * yp / ps, d22 = fac2 / ps, d32 = -yp;
  const double d13 = -(ee * xp / (ps * ps)), d23 = -(ee * yp / (ps * ps)), d33 = ee / ps;
  const double xf = xp / fac2;
  const double fi0 = m_atan2(xf, 1.0) - 2 * kap * (1 + xp * xp * (2 + yp * yp)) * ps;  // atan(xp/fac2)
  const double cf = m_cos(fi0);
  const double co2 = b / (cf * cf);
  const double co1 = co2 / (1 + xf * xf);
  const double fi1 = co1 / fac2 - 4 * kap * co2 * xp * (2 + yp * yp) * ps;
  const double fi2 = -(2 * co1 * xp * yp / (fac2 * fac2)) - 4 * kap * co2 * (xp * xp) * yp * ps;
  const double fi3 = -(2 * kap * co2 * (1 + xp * xp * (2 + yp * yp)));
  const double fi0t = b * m_tan(fi0);
  const double bb2 = fi1 * d12 + fi2 * d22 + fi3 * d32;
  double sq = 1 - 2 * bb2 * y;
  if (sq < 0) return false;
  sq = sqrt(sq);
  const double ynew = 2 * y / (1 + sq);
  const double bb1 = fi1 * d11 + fi2 * d21 + fi3 * d31;
  const double bb3 = fi1 * d13 + fi2 * d23 + fi3 * d33;
  v[0] = x + 0.5 * bb1 * (ynew * ynew);
  v[2] = ynew;
  v[3] = py - fi0t * ynew;
  v[4] = z + 0.5 * beta * bb3 * (ynew * ynew);
  return true;
}

// exact_bend_edge_kick (fringe_mod.f90:1474-1562, no matrix): wedge, dipole fringe, wedge.
BG_COLD void exact_bend_edge(Particle& p, const double* __restrict__ xb, bool entering) {
  const double g_tot = xb[13], beta0 = xb[14];
  const double* q = xb + (entering ? 15 : 18);
  const double edge_angle = q[0], fint = q[1], hgap = q[2];
  double v[6] = {p.x, p.px, p.y, p.py, p.z, p.pz};
  bool ok;
  if (entering)
    ok = wedger(edge_angle, 0.0, v) && fringe_dipoler(v, g_tot, beta0, 1 * fint, hgap, true) &&
         wedger(-edge_angle, g_tot, v);
  else
    ok = wedger(-edge_angle, g_tot, v) && fringe_dipoler(v, g_tot, beta0, 1 * fint, hgap, false) &&
         wedger(edge_angle, 0.0, v);
  if (!ok) {
    p.state = S_LOST_PZ;
    return;
  }
  p.x = v[0];
  p.px = v[1];
  p.y = v[2];
  p.py = v[3];
  p.z = v[4];
}

// track_this_elsep (track_a_thick_multipole.f90:137-240, no matrix): one step through an
// elseparator's transverse electric field in the frame turned by the field angle; false if the
// particle is lost (lost_pz returns it to the element's entrance coordinates, start).
BG_COLD bool elsep_step(Particle& p, const double* __restrict__ xb, double step_len, const Particle& start,
                        const Globals& G) {
  const bool rot = xb[24] != 0;
  if (rot) tilt(p, xb[22], xb[23]);
  const double k_E = xb[25], beta_ref = xb[26];
  const double beta = p.beta, px = p.px, py = p.py, pz = p.pz;
  const double pc = G.p0c * (1 + pz);
  const double E_tot = pc / beta;
  const double E_rel = E_tot / G.p0c;
  const double p_factor = xb[27] + px * px + py * py;
  if (E_rel * E_rel < p_factor) {
    p = start;
    p.state = S_LOST_PZ;
    return false;
  }
  const double ps2 = E_rel * E_rel - p_factor;
  const double ps = sqrt(ps2);
  const double coef = k_E * step_len / ps;
  if (fabs(coef) > 10) {
    p.state = S_LOST;
    return false;
  }
  double sinh_k, cosh_k, cosh1_k;
  const double c2 = coef * coef, c4 = c2 * c2;
  if (fabs(coef) < 1e-3) {
    const double alpha = step_len / ps;
    sinh_k = alpha * (1 + c2 / 6 + c4 / 120);
    cosh1_k = alpha * coef * (1.0 / 2 + c2 / 24 + c4 / 720);
    double sh, ch;
    m_sinhcosh(coef, sh, ch);
    cosh_k = ch / k_E;
  } else {
    double sh, ch;
    m_sinhcosh(coef, sh, ch);
    cosh_k = ch / k_E;
    sinh_k = sh / k_E;
    cosh1_k = cosh_k - 1 / k_E;
  }
  const double dx = E_rel * cosh1_k + px * sinh_k;
  p.x = p.x + dx;
  p.px = k_E * (E_rel * sinh_k + px * cosh_k);
  p.y = p.y + step_len * py / ps;
  const double dct = E_rel * sinh_k + px * cosh1_k;
  p.z = p.z + p.beta * (step_len / beta_ref - dct);
  energy_kick(p, dx * k_E * G.p0c, G);
  refresh(p, G);
  if (rot) tilt(p, xb[22], -xb[23]);
  return true;
}

// One edge of apply_element_edge_kick (apply_element_edge_kick.f90:37-282) for a quadrupole,
// sextupole, octupole or thick multipole with an extra block: the beta check, the electric
// fringe after the magnetic edge at the entrance and before it at the exit, and the hard and
// soft fringes of the quadrupole (hard then soft entering, soft then hard leaving) or sextupole.
BG_COLD void straight_edge(Particle& p, const double* __restrict__ xb, bool entering, const Globals& G) {
  const int bits = (int)xb[entering ? 3 : 4];
  if (!(bits & EX_CALL)) return;
  if (p.beta == 0) p.state = S_LOST;
  if (!entering && (bits & EX_ELEC)) elec_fringe(p, xb, xb[6], G);
  if (entering) {
    if (bits & EX_HARD) hard_edge(p, xb, true);
    if (bits & EX_SOFT) soft_quad_edge(p, xb, true);
  } else {
    if (bits & EX_SOFT) soft_quad_edge(p, xb, false);
    if (bits & EX_HARD) hard_edge(p, xb, false);
  }
  if (bits & EX_ESEP) {  // the elseparator's longitudinal fringe, :263-272
    const double ff = xb[entering ? 28 : 29];
    energy_kick(p, ff * (xb[30] * p.x + xb[31] * p.y), G);
    refresh(p, G);
  }
  if (entering && (bits & EX_ELEC)) elec_fringe(p, xb, xb[5], G);
}

// Electric field of the bend's multipoles (elec_multipole_field.f90:25-60), summed over the
// orders as track_a_bend's apply_multipole_kicks sums it (track_a_bend.f90:384-390).
BG_COLD void elec_field(const Particle& p, const double* __restrict__ e, double& E1, double& E2) {
  const int n_pole = (int)e[0];
  const double* c = e + EL_FIXED;
  const double x = p.x, y = p.y;
  E1 = 0;
  E2 = 0;
  for (int n = 0; n < n_pole; n++) {
    const double b = c[2 * n], a = c[2 * n + 1];
    if (a == 0 && b == 0) continue;
    double ex = 0, ey = 0;
    for (int m = 0; m <= n; m += 2) {
      const double f = BG_CMULTI(n, m) * mexp(x, n - m) * mexp(y, m);
      ex = ex - b * f;
      ey = ey - a * f;
    }
    for (int m = 1; m <= n; m += 2) {
      const double f = BG_CMULTI(n, m) * mexp(x, n - m) * mexp(y, m);
      ex = ex + a * f;
      ey = ey - b * f;
    }
    E1 = E1 + ex;
    E2 = E2 + ey;
  }
}

// The electric kick of track_a_bend's apply_multipole_kicks (track_a_bend.f90:416-432), field
// E1, E2 taken before the magnetic kick; sc = step_len * coef, g the design curvature.
BG_COLD void bend_elec_kick(Particle& p, const double* __restrict__ e, double sc, double g, double E1, double E2,
                            const Globals& G) {
  const double px0 = p.px, py0 = p.py, pz0 = p.pz, z0 = p.z, beta0 = p.beta;
  const double rel_p0 = 1 + pz0;
  const double ps2 = rel_p0 * rel_p0 - px0 * px0 - py0 * py0;
  const double ps = sqrt(ps2) / rel_p0;
  const double f_coef = sc * (1 + g * p.x) * G.charge / (ps * beta0 * G.p0c);
  const double kx = f_coef * E1, ky = f_coef * E2;
  const double alpha = (kx * (2 * px0 + kx) + ky * (2 * py0 + ky)) / (rel_p0 * rel_p0);
  p.px = px0 + kx;
  p.py = py0 + ky;
  p.pz = pz0 + rel_p0 * sqrt_one(alpha);
  const double mp = e[7];
  p.beta = (1 + p.pz) / sqrt(ps2 + p.px * p.px + p.py * p.py + mp * mp);
  p.z = z0 * p.beta / beta0;
  refresh(p, G);
}

// ---- misaligned-bend frame ------------------------------------------------------------------
// offset_particle for a bend with offsets, pitches or z_offset (offset_particle.f90:204-257 set,
// 399-457 unset): the chain of bend_shift, misalignment and ref_tilt transforms of the floor
// position is affine in the particle's (x, y); its rotation part and the translations were
// folded on the host with the reference's own sequence of operations, and the steps acting on
// the position are replayed here in the same order (the bend frame block, table.h). The momentum
// is rotated by the chain's rotation, then the particle drifts to the element's edge.
BG_COLD void bend_frame(Particle& p, const double* __restrict__ m, bool set) {
  const int n_set = (int)m[0];
  const int n = set ? n_set : (int)m[1];
  const double* w = m + (set ? 4 : 13);
  const double* st = m + BF_FIXED + (set ? 0 : BF_STEP * n_set);
  double r[3] = {p.x, p.y, 0.0};
  for (int k = 0; k < n; k++) {
    const double* s = st + BF_STEP * k;
    const int op = (int)s[0];
    if (op & FS_SUB) {
      r[0] = r[0] - s[1];
      r[1] = r[1] - s[2];
      r[2] = r[2] - s[3];
    }
    if (op & FS_SUBZ) r[2] = r[2] - s[3];
    if (op & FS_MAT) {
      double q[3];
      matvec3(s + 4, r, q);
      r[0] = q[0];
      r[1] = q[1];
      r[2] = q[2];
    }
    if (op & FS_ADD) {
      r[0] = r[0] + s[13];
      r[1] = r[1] + s[14];
      r[2] = r[2] + s[15];
    }
    if (op & FS_ADDZ) r[2] = r[2] + s[15];
  }
  const double s_pos = r[2];
  const double rel_p = 1 + p.pz;
  const double pz2 = rel_p * rel_p - p.px * p.px - p.py * p.py;
  if (pz2 <= 0) {
    p.state = S_LOST_PZ;
  } else {
    const double v[3] = {p.px, p.py, 1 * sqrt(pz2)};
    double pv[3];
    matvec3(w, v, pv);
    p.px = pv[0];
    p.py = pv[1];
    p.x = r[0];
    p.y = r[1];
  }
  const double ds = m[set ? 2 : 3] - s_pos;
  if (fabs(ds) > 1e-14 && p.state == S_ALIVE) drift_noref(p, ds);
}

// modulo2 (sim_utils/special_functions/modulo2_mod.f90:85-100): x + 2 n amp in [-amp, amp)
BG_HD double modulo2(double x, double amp) {
  double two = 2 * amp;
  double r = fmod(x, two);
  if (r != 0 && ((r < 0) != (two < 0))) r += two;
  if (r >= amp) r = r - two;
  return r;
}

// RF phase of track_a_rfcavity.f90:78-86 with particle_rf_time (particle_rf_time.f90:89, 115).
// The reference evaluates twopi*(phi0 - t*f) in real(qp) and rounds once; t*f and the
// subtraction are carried here in double-double (exact product by fma, two-sum), then rounded.
BG_HD double rf_phase(const Particle& p, double phi0, double f, double twopi_mp) {
  double time = -p.z / (p.beta * kCLight);
  double amp = 0.5 / f;
  double t_lo = 0;
  if (!(fabs(time) < amp)) {
    // Outside half an RF period the reference folds t into [-amp, amp) with amp = 0.5_qp/f in
    // real(qp), where t - k 2 amp is exact. Kept here as t + t_lo, with amp carried as
    // amp + amp_lo (the residual 0.5 - amp f is exact by fma).
    const double amp_lo = fma(-amp, f, 0.5) / f;
    const double k = floor((time + amp) / (2 * amp));
    const double ph = k * (2 * amp);
    const double pl = fma(k, 2 * amp, -ph);          // k 2 amp = ph + pl exactly
    const double s = time - ph;                      // two-sum of time and -ph
    const double sb = s - time;
    const double e = (time - (s - sb)) + (-ph - sb);
    const double lo = e - pl - k * (2 * amp_lo);
    time = s + lo;
    t_lo = lo - (time - s);
  }
  double pr = time * f;
  double pe = fma(time, f, -pr) + t_lo * f;
  double s = phi0 - pr;
  double bb = s - phi0;
  double err = (phi0 - (s - bb)) + (-pr - bb);
  double lo = err - pe;
  double phase0 = fma(kTwoPi, s, kTwoPi * lo);
  phase0 = phase0 + twopi_mp;
  return modulo2(phase0, kPi);
}

}  // namespace bmadgpu
