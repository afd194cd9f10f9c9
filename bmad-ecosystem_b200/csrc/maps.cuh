// maps.cuh -- FP64 device maps of Bmad's bmad_standard tracking, one particle per thread.
//
// Each function restates one reference routine (cited) on a particle held in registers. The
// element invariants come precomputed from the packed table (lattice.cpp). Quantities that
// depend on the particle only through pz (1/(1+pz), the drift's reference-motion term, the
// low-energy z-correction slope) are cached in the particle and refreshed when the energy
// changes, instead of being recomputed in every element as the reference does. Where an
// identity replaces a transcendental (the exact bend), the comment says so; results agree with
// the reference's operation order to rounding (tested against the oracle to 1e-12).
#pragma once
#include <stdint.h>

#include "table.h"

namespace bmadgpu {

constexpr double kPi = 3.141592653589793238462643383279;
constexpr double kTwoPi = 2 * kPi;
constexpr double kCLight = 2.99792458e8;

enum : int { S_ALIVE = 1, S_LOST = 2, S_NEG_X = 3, S_POS_X = 4, S_NEG_Y = 5, S_POS_Y = 6, S_LOST_PZ = 8 };
enum : int { L_UPSTREAM = 1, L_DOWNSTREAM = 2, L_INSIDE = 3 };

struct Globals {            // branch constants (lat_param_struct / bmad_com)
  double p0c, e_tot, mass, beta0, max_ap;
  double mass2;             // mass^2
  double lez_f, me2;        // low_energy_z_correction: beta0^2 (2 beta0^2 - (m/E)^2/2), (m/E)^2
  double lez_thresh;        // 3e-7 * e_tot
};

struct Particle {
  double x, px, y, py, z, pz, beta;
  int state;
  // cached functions of pz (and beta), refreshed by refresh()
  double inv_rel;           // 1 / (1 + pz)
  double dzb;               // sqrt_one(m^2 (2 pz + pz^2) / ((p0c (1+pz))^2 + m^2)) = beta/beta_ref - 1
  double sq_inv;            // sqrt(1 / (1 + pz))
  double lez;               // low_energy_z_correction per unit length
};

__device__ __forceinline__ double sqrt_one(double x) {  // sim_utils/special_functions/sqrt_one.f90
  double sq = sqrt(1 + x);
  return x / (sq + 1);
}

__device__ __forceinline__ void refresh(Particle& p, const Globals& g) {
  double rel = 1 + p.pz;
  p.inv_rel = 1.0 / rel;
  double pr = g.p0c * rel;
  p.dzb = sqrt_one((g.mass2 * (2 * p.pz + p.pz * p.pz)) / (pr * pr + g.mass2));
  p.sq_inv = sqrt(p.inv_rel);
  // low_energy_z_correction.f90:43-52
  double b0pz = g.beta0 * p.pz;
  if (g.mass * (b0pz * b0pz) < g.lez_thresh) {
    double b02 = g.beta0 * g.beta0;
    p.lez = p.pz * (1 - 3 * (p.pz * b02) / 2 + (p.pz * p.pz) * g.lez_f) * g.me2;
  } else {
    p.lez = (p.beta - g.beta0) / g.beta0;
  }
}

// orbit_too_large, bmad/low_level/orbit_too_large.f90:26-120
__device__ __forceinline__ bool orbit_too_large(Particle& p, const Globals& g) {
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

// check_aperture_limit (rectangular / elliptical branch), check_aperture_limit.f90:286-324
__device__ __forceinline__ void aperture(Particle& p, const ApRec& a, bool elliptical) {
  double xp = p.x, yp = p.y;
  if (elliptical) {
    double rx = xp / a.x2_lim, ry = yp / a.y2_lim;
    double r = rx * rx + ry * ry;
    if (r < 1) return;
    if (fabs(rx) > fabs(ry)) p.state = (xp > 0) ? S_POS_X : S_NEG_X;
    else p.state = (yp > 0) ? S_POS_Y : S_NEG_Y;
    return;
  }
  bool out = (a.x1_lim != 0 && xp < a.x1_lim) || (a.x2_lim != 0 && xp > a.x2_lim) ||
             (a.y1_lim != 0 && yp < a.y1_lim) || (a.y2_lim != 0 && yp > a.y2_lim);
  if (!out) return;
  double uf = 0;
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

// track_a_drift, bmad/low_level/track_a_drift.f90:25-116 (direction = +1, with ref. motion).
// sqrt_one(-pxy2)/ps = -pxy2 / (ps (1 + ps)); the first z term is the cached p.dzb.
__device__ __forceinline__ void drift(Particle& p, double L) {
  if (L == 0) return;
  double px_rel = p.px * p.inv_rel;
  double py_rel = p.py * p.inv_rel;
  double pxy2 = px_rel * px_rel + py_rel * py_rel;
  if (pxy2 >= 1) { p.state = S_LOST_PZ; return; }
  double ps = sqrt(1 - pxy2);
  double r = 1.0 / (ps * (1 + ps));
  double inv_ps = (1 + ps) * r;
  p.x = p.x + L * px_rel * inv_ps;
  p.y = p.y + L * py_rel * inv_ps;
  double dz = (p.beta > 0) ? L * (p.dzb - pxy2 * r) : L * (1 - inv_ps);
  p.z = p.z + dz;
}

// Drift without reference motion (offset_particle.f90:279-282, include_ref_motion = F).
__device__ __forceinline__ void drift_no_ref(Particle& p, double L) {
  double px_rel = p.px * p.inv_rel, py_rel = p.py * p.inv_rel;
  double pxy2 = px_rel * px_rel + py_rel * py_rel;
  if (pxy2 >= 1) { p.state = S_LOST_PZ; return; }
  double ps = sqrt(1 - pxy2);
  p.x = p.x + L * px_rel / ps;
  p.y = p.y + L * py_rel / ps;
  p.z = p.z - L / ps;
}

// Sum of ab_multipole_kick over n < n_pole (multipole_mod.f90:314-401) as one complex Horner
// evaluation: kx - i ky = -sum_n (b_n + i a_n) (x + i y)^n. c = [(b_0, a_0), (b_1, a_1), ...].
__device__ __forceinline__ void multipole_kick_sum(const double* __restrict__ c, int n_pole, double x, double y,
                                                   double& kx, double& ky) {
  double pr = c[2 * (n_pole - 1)], pi = c[2 * (n_pole - 1) + 1];
  for (int n = n_pole - 2; n >= 0; n--) {
    double nr = pr * x - pi * y + c[2 * n];
    double ni = pr * y + pi * x + c[2 * n + 1];
    pr = nr;
    pi = ni;
  }
  kx = -pr;
  ky = pi;
}

// ab_multipole_kicks (multipole_mod.f90:82-121), magnetic, coefficients pre-scaled.
__device__ __forceinline__ void kicks(Particle& p, const double* __restrict__ c, int n_pole) {
  double kx, ky;
  multipole_kick_sum(c, n_pole, p.x, p.y, kx, ky);
  p.px = p.px + kx;
  p.py = p.py + ky;
}

// tilt_coords, bmad/code/tilt_coords.f90:18-53 (cos/sin precomputed)
__device__ __forceinline__ void tilt(Particle& p, double c, double s) {
  double x = p.x, y = p.y, px = p.px, py = p.py;
  p.x = c * x + s * y;
  p.y = -s * x + c * y;
  p.px = c * px + s * py;
  p.py = -s * px + c * py;
}

// offset_particle set/unset for straight elements with x/y offsets and tilt
// (offset_particle.f90:201-330, 374-459 with zero pitches and z_offset: the transforms reduce to
// exact shifts plus the pz-loss test).
__device__ __forceinline__ void offset_set(Particle& p, const double* __restrict__ m, bool has_tilt) {
  if (m[0] != 0 || m[1] != 0) {
    p.x = p.x - m[0];
    p.y = p.y - m[1];
    double rel_p = 1 + p.pz;
    if (rel_p * rel_p - p.px * p.px - p.py * p.py <= 0) p.state = S_LOST_PZ;
  }
  if (has_tilt) tilt(p, m[2], m[3]);
}
__device__ __forceinline__ void offset_unset(Particle& p, const double* __restrict__ m, bool has_tilt) {
  if (has_tilt) tilt(p, m[2], -m[3]);
  if (m[0] != 0 || m[1] != 0) {
    double rel_p = 1 + p.pz;
    if (rel_p * rel_p - p.px * p.px - p.py * p.py <= 0) p.state = S_LOST_PZ;
    p.x = p.x + m[0];
    p.y = p.y + m[1];
  }
}

// sinh and cosh of a non-negative argument from one expm1.
__device__ __forceinline__ void sinh_cosh(double a, double& sh, double& ch) {
  double em = expm1(a);
  double ep = em + 1;
  double inv = 1.0 / ep;
  sh = 0.5 * em * (1 + inv);
  ch = 1 + 0.5 * em * em * inv;
}

// One body step of track_a_quadrupole (track_a_quadrupole.f90:95-120) with quad_mat2_calc
// (quad_mat2_calc.f90:22-61) for both planes. b1_l = b1/L, sqrt_bl = sqrt(|b1/L|).
__device__ __forceinline__ void quad_step(Particle& p, double b1_l, double sqrt_bl, double step_len) {
  double k1 = b1_l * p.inv_rel;             // k1 = b1 / (L (1 + pz))
  double sqrt_k = sqrt_bl * p.sq_inv;
  double sk_l = sqrt_k * step_len;
  double cx, sx, cy, sy;                    // x plane uses -k1, y plane +k1
  if (fabs(sk_l) < 1e-10) {
    double k_l2 = k1 * (step_len * step_len);
    cx = 1 - k_l2 / 2;
    sx = (1 - k_l2 / 6) * step_len;
    cy = 1 + k_l2 / 2;
    sy = (1 + k_l2 / 6) * step_len;
  } else {
    double st, ct, sh, ch;
    sincos(sk_l, &st, &ct);
    sinh_cosh(sk_l, sh, ch);
    double inv_sk = 1.0 / sqrt_k;
    if (k1 > 0) {           // x focusing (-k1 < 0), y defocusing
      cx = ct; sx = st * inv_sk; cy = ch; sy = sh * inv_sk;
    } else {
      cx = ch; sx = sh * inv_sk; cy = ct; sy = st * inv_sk;
    }
  }
  double ir = p.inv_rel;
  double ir2 = ir * ir;
  double zx0 = -k1 * (-cx * sx + step_len) / 4, zx1 = k1 * (sx * sx) * ir / 2, zx2 = -(cx * sx + step_len) * ir2 / 4;
  double zy0 = k1 * (-cy * sy + step_len) / 4, zy1 = -k1 * (sy * sy) * ir / 2, zy2 = -(cy * sy + step_len) * ir2 / 4;
  double x = p.x, px = p.px, y = p.y, py = p.py;
  p.z = p.z + (zx0 * (x * x) + zx1 * x * px + zx2 * (px * px) + zy0 * (y * y) + zy1 * y * py + zy2 * (py * py));
  p.x = cx * x + sx * ir * px;
  p.px = -b1_l * sx * x + cx * px;          // mat2(2,1) = k sx rel_p with k = -k1
  p.y = cy * y + sy * ir * py;
  p.py = b1_l * sy * y + cy * py;
  p.z = p.z + step_len * p.lez;
}

// hwang_bend_edge_kick, bmad/modules/fringe_mod.f90:241-419 (time_dir = +1).
// e: [gt, gt2, gs2, k1_tane, fg_factor, g_tot, gt*g_tot*(1 + 2 tan_e^2)]
__device__ __forceinline__ void hwang_edge(Particle& p, const double* __restrict__ e, bool entering) {
  double gt = e[0], gt2 = e[1], gs2 = e[2], k1t = e[3], fg = e[4], gtot = e[5], cdpx = e[6];
  double ef = p.inv_rel;
  double v1 = p.x, v2 = p.px, v3 = p.y, v4 = p.py;
  double v11 = v1 * v1, v33 = v3 * v3;
  double dx, dpx, dy, dpy, dz;
  if (entering) {
    dx = (-gt2 * v11 + gs2 * v33) * ef / 2;
    dpx = (cdpx * v33 / 2 + gt2 * (v1 * v2 - v3 * v4) + k1t * (v11 - v33)) * ef;
    dy = gt2 * v1 * v3 * ef;
    dpy = (fg * v3 - gt2 * v1 * v4 - (gtot + gt2) * v2 * v3 - 2 * k1t * v1 * v3) * ef;
    dz = (ef * ef) * 0.5 *
         (v33 * fg + (v11 * v1) * (4.0 * k1t - gt * gt2) / 6.0 + 0.5 * v1 * v33 * (-4.0 * k1t + gt * gs2) +
          (v11 * v2 - 2.0 * v1 * v3 * v4) * gt2 - v2 * v33 * gs2);
  } else {
    dx = (gt2 * v11 - gs2 * v33) * ef / 2;
    dpx = (gt2 * (v3 * v4 - v1 * v2) + k1t * (v11 - v33) - gt * gt2 * (v11 + v33) / 2) * ef;
    dy = -gt2 * v1 * v3 * ef;
    dpy = (fg * v3 + gt2 * v1 * v4 + (gtot + gt2) * v2 * v3 + (gt * gs2 - 2 * k1t) * v1 * v3) * ef;
    dz = (ef * ef) * 0.5 *
         (v33 * fg + (v11 * v1) * (4.0 * k1t - gt * gt2) / 6.0 + 0.5 * v1 * v33 * (-4.0 * k1t + gt * gs2) -
          (v11 * v2 - 2.0 * v1 * v3 * v4) * gt2 + v2 * v33 * gs2);
  }
  p.x = v1 + dx;
  p.px = v2 + (dpx + gt * v1);
  p.y = v3 + dy;
  p.py = v4 + (dpy - gt * v3);
  p.z = p.z + dz;
}

// sbend_body_with_k1_map, track_a_bend.f90:500-659 (ending coordinates only)
__device__ __forceinline__ void bend_k1_step(Particle& p, const double* __restrict__ b) {
  double length = b[0], g = b[1], g_tot = b[2], k1 = b[10];   // k1 = b1 / L
  double rel_p = 1 + p.pz, rel_p2 = rel_p * rel_p;
  double k_x = k1 + g * g_tot;
  double x_c = (g * rel_p - g_tot) / k_x;
  double om_x = sqrt(fabs(k_x) / rel_p), om_y = sqrt(fabs(k1) / rel_p);
  double tau_x = k_x > 0 ? -1.0 : 1.0, tau_y = k1 > 0 ? 1.0 : -1.0;
  if (k_x == 0) tau_x = -1.0;
  if (k1 == 0) tau_y = 1.0;
  double s_x, c_x, z2, s_y, c_y, arg = om_x * length;
  if (arg < 1e-6) {
    s_x = (1 + tau_x * (arg * arg) / 6) * length; c_x = 1 + tau_x * (arg * arg) / 2; z2 = g * (length * length) / (2 * rel_p);
  } else if (k_x > 0) {
    double s, c; sincos(arg, &s, &c); s_x = s / om_x; c_x = c; z2 = tau_x * g * (1 - c_x) / (rel_p * (om_x * om_x));
  } else {
    double s, c; sinh_cosh(arg, s, c); s_x = s / om_x; c_x = c; z2 = tau_x * g * (1 - c_x) / (rel_p * (om_x * om_x));
  }
  arg = om_y * length;
  if (arg < 1e-6) {
    s_y = (1 + tau_y * (arg * arg) / 6) * length; c_y = 1 + tau_y * (arg * arg) / 2;
  } else if (k1 < 0) {
    double s, c; sincos(arg, &s, &c); s_y = s / om_y; c_y = c;
  } else {
    double s, c; sinh_cosh(arg, s, c); s_y = s / om_y; c_y = c;
  }
  double r1 = p.x - x_c, r2 = p.px, r3 = p.y, r4 = p.py;
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
  p.z = p.z + z0 + z1 * r1 + z2 * r2 + z11 * (r1 * r1) + z12 * r1 * r2 + z22 * (r2 * r2) + z33 * (r3 * r3) +
        z34 * r3 * r4 + z44 * (r4 * r4);
}

// Exact sbend body step, track_a_bend.f90:121-209. Returns false if the particle was lost.
// phi_1 = asin(px/pt) and theta = atan2(L_u, -L_v) enter only through their sines and cosines
// except in sinc(angle_p/2); angle_p/2 = angle + phi_1 - theta is recovered as asin of its sine.
__device__ __forceinline__ bool bend_exact_step(Particle& p, const double* __restrict__ b, const Globals& G) {
  double step_len = b[0], g = b[1], g_tot = b[2], dg = b[3], angle = b[4];
  double cos_a = b[5], sin_a = b[6], sinc_a = b[7], cosc_a = b[8], gl2_sincc = b[9];
  double x = p.x, px = p.px, y = p.y, py = p.py, z = p.z, pz = p.pz;
  double rel_p = 1 + pz;
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
  double pt = sqrt(rel_p * rel_p - py * py);
  if (fabs(px) > pt) { p.state = S_LOST_PZ; return false; }
  double inv_pt = 1.0 / pt;
  double g_p = g_tot * inv_pt;
  double s1 = px * inv_pt;                        // sin(phi_1)
  double c1 = sqrt((1 - s1) * (1 + s1));          // cos(phi_1) >= 0
  double cos_plus = cos_a * c1 - sin_a * s1;      // cos(angle + phi_1)
  double sin_plus = sin_a * c1 + cos_a * s1;      // sin(angle + phi_1)
  double ls = (1 + g * x) * step_len * sinc_a;
  double alpha = 2 * sin_plus * ls - g_p * (ls * ls);
  double r = cos_plus * cos_plus + g_p * alpha;
  if (r < 0 || (fabs(g_p) < 1e-5 && fabs(cos_plus) < 1e-5)) {
    p.state = S_LOST;
    p.x = 2 * G.max_ap;
    return false;
  }
  double rad = sqrt(r);
  double xi = (cos_plus > 0) ? alpha / (rad + cos_plus) : (rad - cos_plus) / g_p;
  double x_new = x * cos_a - (step_len * step_len) * g * cosc_a + xi;
  p.x = x_new;
  if (fabs(x_new) > G.max_ap) { p.state = S_LOST; return false; }
  double L_u = xi;
  double L_v = -(step_len * sinc_a + x * sin_a);
  double L_c = sqrt(L_v * L_v + L_u * L_u);
  double inv_lc = 1.0 / L_c;
  double st = L_u * inv_lc, ct = -L_v * inv_lc;   // sin, cos of theta = atan2(L_u, -L_v)
  double sin_u = sin_plus * ct - cos_plus * st;   // sin(angle_p / 2)
  double u;
  if (fabs(sin_u) < 0.7) {
    u = asin(sin_u);
  } else {
    u = angle + asin(s1) - atan2(L_u, -L_v);
  }
  double sinc_u = (fabs(u) < 1e-8) ? 1.0 : sin(u) / u;
  double L_p = L_c / sinc_u;
  double s2t = 2 * st * ct, c2t = (ct - st) * (ct + st);
  p.px = pt * (s2t * cos_plus - c2t * sin_plus);  // pt sin(phi_1 + angle - angle_p)
  p.y = y + py * L_p * inv_pt;
  p.z = z + p.beta * step_len / G.beta0 - rel_p * L_p * inv_pt;
  return true;
}

// apply_energy_kick, bmad/low_level/apply_energy_kick.f90:23-74
__device__ __forceinline__ void energy_kick(Particle& p, double dE, const Globals& G) {
  double pc = (1 + p.pz) * G.p0c;
  double beta_old = p.beta;
  double E_old = pc / p.beta;
  double E_new = E_old + dE;
  if (E_new < G.mass) {
    p.pz = -1;
    p.beta = 0;
    p.state = S_LOST_PZ;
    return;
  }
  p.pz = p.pz + (1 + p.pz) * sqrt_one((2 * E_old * dE + dE * dE) / (pc * pc));
  double pc_new = G.p0c * (1 + p.pz);
  double beta_new = pc_new / E_new;
  p.z = p.z * beta_new / beta_old;
  p.beta = beta_new;
}

// modulo2 (sim_utils/special_functions/modulo2_mod.f90:85-100): x + 2 n amp in [-amp, amp)
__device__ __forceinline__ double modulo2(double x, double amp) {
  double two = 2 * amp;
  double r = fmod(x, two);
  if (r != 0 && ((r < 0) != (two < 0))) r += two;
  if (r >= amp) r = r - two;
  return r;
}

// RF phase of track_a_rfcavity.f90:78-86 with particle_rf_time (relative time). The reference
// evaluates twopi*(phi0 - t*f) in real(qp) and rounds once; here t*f and the subtraction are
// carried in double-double so the rounded result matches.
__device__ __forceinline__ double rf_phase(const Particle& p, double phi0, double f, double twopi_mp) {
  double time = -p.z / (p.beta * kCLight);
  double amp = 0.5 / f;
  if (!(fabs(time) < amp)) time = modulo2(time, amp);
  double pr = time * f;
  double pe = fma(time, f, -pr);
  double s = phi0 - pr;                           // two-sum of phi0 and -pr
  double bb = s - phi0;
  double err = (phi0 - (s - bb)) + (-pr - bb);
  double lo = err - pe;
  double phase0 = fma(kTwoPi, s, kTwoPi * lo);
  phase0 = phase0 + twopi_mp;
  return modulo2(phase0, kPi);
}

}  // namespace bmadgpu
