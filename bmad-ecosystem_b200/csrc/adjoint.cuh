// adjoint.cuh -- hand-written reverse-mode derivatives (vector-Jacobian products) of the element
// maps in maps.cuh / elements.cuh, for d(loss)/d(element strengths).
//
// State: (x, px, y, py, z, pz, beta). beta is carried as a coordinate of its own because the
// maps use the tracked coord%beta (exact bend z, energy kick, RF time, low-energy z), not a
// function of pz. Each vjp_* takes the primitive's INPUT particle (caches refreshed), and maps the
// cotangent of its output (Adj) to the cotangent of its input in place. Branches follow the
// forward map's branch at that input; the aperture and orbit checks are piecewise constant and
// contribute nothing. Parameter cotangents are returned as "scale" derivatives: for a set of
// coefficients c that all scale with one strength k (b1 = k1 L and the multipoles of a quadrupole;
// b_n = k_n L / n! and scaled multipoles of a sextupole/octupole), dL/dk = sum_c c dL/dc / k.
//
// The Jacobians restate, in reverse form, the make_matrix branches of the reference maps:
// track_a_drift.f90:94-114, track_a_quadrupole.f90:204-223 with quad_mat2_calc.f90:65-79,
// track_a_bend.f90:211-300, multipole_mod.f90:123-126, apply_energy_kick.f90:57-69.
#pragma once
#include "elements.cuh"

namespace bmadgpu {

struct Adj {
  double x, px, y, py, z, pz, beta;
};

// Elements with more body steps (or RF slices) than this are outside the adjoint path.
constexpr int kAdjMaxSteps = 16;

// d(dzb)/d(pz): dzb = beta(pz)/beta0 - 1, dbeta/dpz = p0c m^2 / E^3.
BG_HD double d_dzb(double pz, const Globals& G) {
  double P = G.p0c * (1 + pz);
  double E2 = P * P + G.mass2;
  double E = sqrt(E2);
  return G.p0c * G.mass2 / (G.beta0 * E2 * E);
}

// z += low_energy_z(p, ds): cotangents to pz (series branch) or beta.
BG_HD void vjp_lez(const Particle& p, double ds, Adj& a, const Globals& G) {
  if (p.lez_series) {
    double dlez = -3 * G.lez_b02 / 2 + 2 * p.pz * G.lez_f;
    a.pz += a.z * ds * G.lez_me2 * (p.lez_a + p.pz * dlez);
  } else {
    a.beta += a.z * ds / G.beta0;
  }
}

// track_a_drift
BG_HD void vjp_drift(const Particle& p, double L, Adj& a, const Globals& G) {
  if (L == 0) return;
  double rel = 1 + p.pz;
  double ar = p.px / rel, br = p.py / rel;
  double s2 = ar * ar + br * br;
  double ps = sqrt(1 - s2);
  double ips = 1 / ps, ips3 = ips * ips * ips;
  double abar = a.x * L * (ips + ar * ar * ips3) + a.y * L * (ar * br * ips3) - a.z * L * ar * ips3;
  double bbar = a.x * L * (ar * br * ips3) + a.y * L * (ips + br * br * ips3) - a.z * L * br * ips3;
  a.px += abar / rel;
  a.py += bbar / rel;
  a.pz += -(abar * ar + bbar * br) / rel;
  if (p.beta > 0) a.pz += a.z * L * d_dzb(p.pz, G);
}

// Derivatives of quad_mat2_calc's cx, sx with respect to k (quad_mat2_calc.f90:34-47).
BG_HD void quad_cs_dk(double k, double l, double cx, double sx, double& dcx, double& dsx) {
  double skl = sqrt(fabs(k)) * l;
  dcx = l * sx / 2;
  if (fabs(skl) < 1e-10) {
    dcx = l * l / 2;
    dsx = l * l * l / 6;
    return;
  }
  double u = k * l * l;
  if (fabs(u) < 0.1) {
    // l^3 sum_{n>=1} n u^(n-1) / (2n+1)!, to u^4
    dsx = l * l * l * (1.0 / 6 + u * (2.0 / 120 + u * (3.0 / 5040 + u * (4.0 / 362880 + u * (5.0 / 39916800)))));
  } else {
    dsx = (l * cx - sx) / (2 * k);
  }
}

// Cotangent of (k, rel) from the cotangents of one plane's quad_mat2 outputs.
// lc: cotangent of cx (m11 and m22), l12, l21, lz0, lz1, lz2.
BG_HD void quad_mat2_vjp(double k, double l, double rel, double lc, double l12, double l21, double lz0, double lz1,
                         double lz2, double& gk, double& grel) {
  double sk = sqrt(fabs(k)), skl = sk * l;
  double cx, sx;
  if (fabs(skl) < 1e-10) {
    double k_l2 = k * (l * l);
    cx = 1 + k_l2 / 2;
    sx = (1 + k_l2 / 6) * l;
  } else if (k < 0) {
    cx = cos(skl);
    sx = sin(skl) / sk;
  } else {
    cx = cosh(skl);
    sx = sinh(skl) / sk;
  }
  double dcx, dsx;
  quad_cs_dk(k, l, cx, sx, dcx, dsx);
  // m12 = sx/rel, m21 = k sx rel, z0 = k(l - cx sx)/4, z1 = -k sx^2/(2 rel), z2 = -(cx sx + l)/(4 rel^2)
  double d_cs = dcx * sx + cx * dsx;
  gk = lc * dcx + l12 * dsx / rel + l21 * (sx + k * dsx) * rel + lz0 * ((l - cx * sx) / 4 - k * d_cs / 4) +
       lz1 * (-(sx * sx + 2 * k * sx * dsx) / (2 * rel)) + lz2 * (-d_cs / (4 * rel * rel));
  grel = l12 * (-sx / (rel * rel)) + l21 * k * sx + lz1 * (k * sx * sx / (2 * rel * rel)) +
         lz2 * ((cx * sx + l) / (2 * rel * rel * rel));
}

// One quad body step (quad_step); gb1 += d/d(b1) contribution times b1 (scale form).
BG_HD void vjp_quad_step(const Particle& p, double b1, double length, double sl, Adj& a, double& gscale,
                         const Globals& G) {
  double rel = 1 + p.pz;
  double k1 = b1 / (length * rel);
  double ax, bx, cx_, dx, zx0, zx1, zx2, ay, by, cy, dy, zy0, zy1, zy2;
  const double ef = 1 / rel;
  quad_mat2(-k1, sl, rel, ef, ax, bx, cx_, dx, zx0, zx1, zx2);
  quad_mat2(k1, sl, rel, ef, ay, by, cy, dy, zy0, zy1, zy2);
  double x = p.x, px = p.px, y = p.y, py = p.py;
  // low_energy_z on the stepped particle: pz and beta are unchanged by the step
  vjp_lez(p, sl, a, G);
  Adj o = a;
  a.x = o.x * ax + o.px * cx_ + o.z * (2 * zx0 * x + zx1 * px);
  a.px = o.x * bx + o.px * dx + o.z * (zx1 * x + 2 * zx2 * px);
  a.y = o.y * ay + o.py * cy + o.z * (2 * zy0 * y + zy1 * py);
  a.py = o.y * by + o.py * dy + o.z * (zy1 * y + 2 * zy2 * py);
  // coefficient cotangents (m11 = m22 = c)
  double gkx, grx, gky, gry;
  quad_mat2_vjp(-k1, sl, rel, o.x * x + o.px * px, o.x * px, o.px * x, o.z * x * x, o.z * x * px, o.z * px * px, gkx,
                grx);
  quad_mat2_vjp(k1, sl, rel, o.y * y + o.py * py, o.y * py, o.py * y, o.z * y * y, o.z * y * py, o.z * py * py, gky,
                gry);
  double gk1 = -gkx + gky;
  double grel = grx + gry + gk1 * (-k1 / rel);
  a.pz += grel;
  gscale += gk1 * k1;  // k1 is proportional to b1: b1 dL/db1 = k1 dL/dk1
}

// ab_multipole_kicks with pre-scaled coefficients c = (b_n, a_n): px += kx, py += ky.
BG_HD void vjp_ab_kicks(const Particle& p, const double* __restrict__ c, int n_pole, Adj& a, double& gscale) {
  const double x = p.x, y = p.y;
  double kx = 0, ky = 0, kxx = 0, kxy = 0, kyx = 0, kyy = 0;
  for (int n = 0; n < n_pole; n++) {
    const double b = c[2 * n], aa = c[2 * n + 1];
    if (b == 0 && aa == 0) continue;
    for (int m = 0; m <= n; m++) {
      double cm = BG_CMULTI(n, m);
      double f = cm * mexp(x, n - m) * mexp(y, m);
      double fx = (n - m > 0) ? cm * (n - m) * mexp(x, n - m - 1) * mexp(y, m) : 0.0;
      double fy = (m > 0) ? cm * m * mexp(x, n - m) * mexp(y, m - 1) : 0.0;
      double cxk, cyk;  // coefficient of f in kx and ky
      if (m % 2 == 0) {
        cxk = b;
        cyk = -aa;
      } else {
        cxk = aa;
        cyk = b;
      }
      kx += cxk * f;
      ky += cyk * f;
      kxx += cxk * fx;
      kxy += cxk * fy;
      kyx += cyk * fx;
      kyy += cyk * fy;
    }
  }
  gscale += a.px * kx + a.py * ky;
  a.x += a.px * kxx + a.py * kyx;
  a.y += a.px * kxy + a.py * kyy;
}

// tilt (rotation by (c, s)); the inverse rotation passes -s.
BG_HD void vjp_tilt(double c, double s, Adj& a) {
  double ax = a.x, ay = a.y, apx = a.px, apy = a.py;
  a.x = c * ax - s * ay;
  a.y = s * ax + c * ay;
  a.px = c * apx - s * apy;
  a.py = s * apx + c * apy;
}

// Exact sbend body step (bend_exact_step).
BG_HD void vjp_bend_exact(const Particle& p, const double* __restrict__ b, Adj& a, const Globals& G) {
  double l = b[0], g = b[1], g_tot = b[2], dg = b[3], angle = b[4];
  double cos_a = b[5], sin_a = b[6], sinc_a = b[7], cosc_a = b[8], gl2_sincc = b[9];
  double x = p.x, px = p.px, py = p.py, pz = p.pz;
  double rel = 1 + pz;
  if (dg == 0 && fabs(x * g) < 1e-9 && fabs(px) < 1e-9 && fabs(py) < 1e-9 && fabs(pz) < 1e-9) {
    double rpp = rel * G.p0c;
    double den = rpp * rpp + G.mass2;
    double gam2 = G.mass2 / den;
    double m56 = l * (gam2 - gl2_sincc);
    double dm56 = l * (-G.mass2 * 2 * rpp * G.p0c / (den * den));
    Adj o = a;
    a.x = o.x * cos_a + o.px * (-g * sin_a) + o.z * (-g * l * sinc_a);
    a.px = o.x * l * sinc_a + o.px * cos_a + o.z * (-g * l * l * cosc_a);
    a.py = o.py + o.y * l;
    a.pz = o.pz + o.x * g * l * l * cosc_a + o.px * g * l * sinc_a + o.z * (m56 + dm56 * pz);
    return;
  }
  // forward intermediates
  double pt = sqrt(rel * rel - py * py);
  double g_p = g_tot / pt;
  double u = px / pt;
  double phi_1 = asin(u);
  double cp = cos(angle + phi_1), sp = sin(angle + phi_1);
  double gx1 = 1 + g * x;
  double ls = gx1 * l * sinc_a;
  double alpha = 2 * gx1 * sp * l * sinc_a - g_p * (ls * ls);
  double r = cp * cp + g_p * alpha;
  double rad = sqrt(r);
  double xi, den = 0;
  if (cp > 0) {
    den = rad + cp;
    xi = alpha / den;
  } else {
    xi = (rad - cp) / g_p;
  }
  double L_u = xi;
  double L_v = -1 * (l * sinc_a + x * sin_a);
  double L_c = sqrt(L_v * L_v + L_u * L_u);
  double theta = atan2(L_u, -L_v);
  double angle_p = 2 * (angle + phi_1 - theta);
  double hp = angle_p / 2;
  double S = 1, dS = 0;
  if (fabs(hp) >= 1e-8) {
    S = sin(hp) / hp;
    dS = (hp * cos(hp) - sin(hp)) / (hp * hp);
  }
  double L_p = L_c / S;
  double psi = phi_1 + angle - angle_p;
  // reverse sweep
  double b_pt = 0, b_rel = 0, b_Lp = 0, b_phi = 0, b_angp = 0, b_Lc = 0, b_Lu = 0, b_Lv = 0, b_xi = 0;
  double b_alpha = 0, b_rad = 0, b_cp = 0, b_sp = 0, b_gp = 0, b_gx1 = 0, b_ls = 0;
  double b_x = 0, b_px = 0, b_py = 0;
  // z' = z + beta l / beta0 - rel L_p / pt
  double beta_bar = a.beta + a.z * l / G.beta0;
  b_rel += -a.z * L_p / pt;
  b_Lp += -a.z * rel / pt;
  b_pt += a.z * rel * L_p / (pt * pt);
  // y' = y + py L_p / pt
  b_py += a.y * L_p / pt;
  b_Lp += a.y * py / pt;
  b_pt += -a.y * py * L_p / (pt * pt);
  // px' = pt sin(psi)
  b_pt += a.px * sin(psi);
  double b_psi = a.px * pt * cos(psi);
  b_phi += b_psi;
  b_angp += -b_psi;
  // py' = py, pz' = pz
  b_py += a.py;
  double b_pz = a.pz;
  // L_p = L_c / S(hp)
  b_Lc += b_Lp / S;
  double b_S = -b_Lp * L_c / (S * S);
  b_angp += b_S * dS / 2;
  // angle_p = 2 (angle + phi_1 - theta)
  b_phi += 2 * b_angp;
  double b_theta = -2 * b_angp;
  double X = -L_v, Y = L_u, R2 = X * X + Y * Y;
  b_Lu += b_theta * X / R2;
  double b_X = -b_theta * Y / R2;
  b_Lv += -b_X;
  // L_c = sqrt(L_v^2 + L_u^2)
  b_Lv += b_Lc * L_v / L_c;
  b_Lu += b_Lc * L_u / L_c;
  // L_v = -(l sinc_a + x sin_a), L_u = xi
  b_x += -b_Lv * sin_a;
  b_xi += b_Lu;
  // x' = x cos_a - l^2 g cosc_a + xi
  b_x += a.x * cos_a;
  b_xi += a.x;
  // xi
  if (cp > 0) {
    b_alpha += b_xi / den;
    double b_den = -b_xi * alpha / (den * den);
    b_rad += b_den;
    b_cp += b_den;
  } else {
    b_rad += b_xi / g_p;
    b_cp += -b_xi / g_p;
    b_gp += -b_xi * (rad - cp) / (g_p * g_p);
  }
  // rad = sqrt(r); r = cp^2 + g_p alpha
  double b_r = b_rad / (2 * rad);
  b_cp += b_r * 2 * cp;
  b_gp += b_r * alpha;
  b_alpha += b_r * g_p;
  // alpha = 2 gx1 sp l sinc_a - g_p ls^2; ls = gx1 l sinc_a
  b_gx1 += b_alpha * 2 * sp * l * sinc_a;
  b_sp += b_alpha * 2 * gx1 * l * sinc_a;
  b_gp += -b_alpha * ls * ls;
  b_ls += -b_alpha * g_p * 2 * ls;
  b_gx1 += b_ls * l * sinc_a;
  b_x += b_gx1 * g;
  // cp, sp of angle + phi_1
  b_phi += -b_cp * sp + b_sp * cp;
  // phi_1 = asin(px/pt)
  double b_u = b_phi / sqrt(1 - u * u);
  b_px += b_u / pt;
  b_pt += -b_u * px / (pt * pt);
  // g_p = g_tot / pt
  b_pt += -b_gp * g_tot / (pt * pt);
  // pt = sqrt(rel^2 - py^2)
  b_rel += b_pt * rel / pt;
  b_py += -b_pt * py / pt;
  b_pz += b_rel;
  a.x = b_x;
  a.px = b_px;
  a.py = b_py;
  a.pz = b_pz;
  a.beta = beta_bar;
  // a.y and a.z pass through (y' = y + ..., z' = z + ...)
}

// apply_energy_kick: (pz, beta, z) with energy gain dE; g_dE receives dL/d(dE).
BG_HD void vjp_energy_kick(const Particle& p, double dE, Adj& a, double& g_dE, const Globals& G) {
  double p0c = G.p0c;
  double rel = 1 + p.pz;
  double pc = rel * p0c;
  double beta = p.beta;
  double E_old = pc / beta;
  double E_new = E_old + dE;
  double A = (2 * E_old * dE + dE * dE) / (pc * pc);
  double S = sqrt(1 + A);
  double pz_new = p.pz + rel * sqrt_one(A);
  double pc_new = p0c * (1 + pz_new);
  double beta_new = pc_new / E_new;
  // z' = z beta_new / beta
  double b_z = a.z * beta_new / beta;
  double b_bnew = a.beta + a.z * p.z / beta;
  double b_beta = -a.z * p.z * beta_new / (beta * beta);
  // beta_new = p0c (1 + pz_new) / E_new
  double b_pznew = a.pz + b_bnew * p0c / E_new;
  double b_Enew = -b_bnew * beta_new / E_new;
  // 1 + pz_new = rel S(A), A(E_old, dE, pc)
  double b_rel = b_pznew * S;
  double b_A = b_pznew * rel / (2 * S);
  double b_Eold = b_A * 2 * dE / (pc * pc) + b_Enew;
  double b_dE = b_A * 2 * E_new / (pc * pc) + b_Enew;
  double b_pc = b_A * (-2 * A / pc);
  // E_old = pc / beta
  b_pc += b_Eold / beta;
  b_beta += -b_Eold * pc / (beta * beta);
  b_rel += b_pc * p0c;
  a.z = b_z;
  a.pz = b_rel;
  a.beta = b_beta;
  g_dE += b_dE;
}

// Tape of sub-step inputs inside one element.
struct AdjTape {
  Particle in[2 * kAdjMaxSteps + 6];
  int n = 0;
  BG_HD void push(const Particle& p) { in[n++] = p; }
};

#if defined(__CUDACC__)
#define BG_HOST_DEVICE __host__ __device__ inline
#else
#define BG_HOST_DEVICE inline
#endif

// Which element bodies the adjoint covers (elements.cuh forms). 0 if supported.
BG_HOST_DEVICE int adj_supported(const EleHdr& h) {
  if (h.flags & (F_PITCH | F_EXTRA)) return 1;  // pitched / bend-frame misalignment, electric
                                                // multipoles, higher-order edges: no
                                                // vector-Jacobian product written
  switch (h.kind) {
    case K_MARKER:
    case K_DRIFT:
      return 0;
    case K_QUAD:
    case K_THICK:
      return h.n_step <= kAdjMaxSteps ? 0 : 1;
    case K_SBEND:
      if (h.flags & (F_EDGE_IN | F_EDGE_OUT | F_BEND_K1)) return 1;
      if (h.n_pole) return 1;
      return h.n_step <= kAdjMaxSteps ? 0 : 1;
    case K_RFCAV:
      return h.n_step <= kAdjMaxSteps ? 0 : 1;
    default:
      return 1;  // thin multipoles
  }
}

// Reverse of one element body (the part between track1's checks) at input p (caches refreshed):
// maps the cotangent of the element's output to that of its input; gscale += sum_c c dL/dc over
// the element's strength coefficients.
BG_HD void vjp_element(const EleHdr& h, const double* __restrict__ pool, const Particle& pin, Adj& a,
                       double& gscale, const Globals& G) {
  const double* b = pool + h.param;
  Particle p = pin;
  switch (h.kind) {
    case K_DRIFT:
      vjp_drift(p, b[0], a, G);
      return;
    case K_QUAD: {
      const int np = h.n_pole, n_step = h.n_step;
      const double* kh = b + 3;
      const double* kf = kh + 2 * np;
      const double* mis = b + 3 + 4 * np;
      const bool has_t = h.flags & F_TILT, misal = h.flags & F_MISALIGN;
      const double b1 = b[0], length = b[1], sl = b[2];
      AdjTape t;
      if (misal) offset_set(p, mis, has_t);
      for (int i = 0; i <= n_step; i++) {
        if (i > 0) {
          t.push(p);
          quad_step(p, b1, length, sl, G);
        }
        if (np) {
          t.push(p);
          ab_kicks(p, (i == 0 || i == n_step) ? kh : kf, np);
        }
      }
      if (misal && has_t) vjp_tilt(mis[2], -mis[3], a);
      for (int i = n_step; i >= 0; i--) {
        if (np) vjp_ab_kicks(t.in[--t.n], (i == 0 || i == n_step) ? kh : kf, np, a, gscale);
        if (i > 0) vjp_quad_step(t.in[--t.n], b1, length, sl, a, gscale, G);
      }
      if (misal && has_t) vjp_tilt(mis[2], mis[3], a);
      return;
    }
    case K_THICK: {
      const int np = h.n_pole, n_step = h.n_step;
      const double* kh = b + 1;
      const double* kf = kh + 2 * np;
      const double* mis = b + 1 + 4 * np;
      const bool has_t = h.flags & F_TILT, misal = h.flags & F_MISALIGN;
      const double sl = b[0];
      AdjTape t;
      if (misal) offset_set(p, mis, has_t);
      for (int i = 0; i <= n_step; i++) {
        if (i > 0) {
          t.push(p);
          drift(p, sl);
        }
        if (np) {
          t.push(p);
          ab_kicks(p, (i == 0 || i == n_step) ? kh : kf, np);
        }
      }
      if (misal && has_t) vjp_tilt(mis[2], -mis[3], a);
      for (int i = n_step; i >= 0; i--) {
        if (np) vjp_ab_kicks(t.in[--t.n], (i == 0 || i == n_step) ? kh : kf, np, a, gscale);
        if (i > 0) vjp_drift(t.in[--t.n], sl, a, G);
      }
      if (misal && has_t) vjp_tilt(mis[2], mis[3], a);
      return;
    }
    case K_SBEND: {
      const double* mis = b + SB_FIXED;
      const bool misal = h.flags & F_MISALIGN;
      AdjTape t;
      if (misal) tilt(p, mis[2], mis[3]);
      for (int n = 1; n <= h.n_step; n++) {
        t.push(p);
        if (h.flags & F_BEND_DRIFT) drift(p, b[0]);
        else bend_exact_step(p, b, G);
      }
      if (misal) vjp_tilt(mis[2], -mis[3], a);
      for (int n = h.n_step; n >= 1; n--) {
        const Particle& q = t.in[--t.n];
        if (h.flags & F_BEND_DRIFT) vjp_drift(q, b[0], a, G);
        else vjp_bend_exact(q, b, a, G);
      }
      if (misal) vjp_tilt(mis[2], mis[3], a);
      return;
    }
    case K_RFCAV: {
      const int np = h.n_pole;
      const double* kh = b + RF_FIXED;
      const double* mis = kh + 2 * np;
      const bool has_t = h.flags & F_TILT, misal = h.flags & F_MISALIGN;
      const double voltage = b[0], f = b[1], slice_len = b[4];
      const int n_slice = h.n_step;
      if (misal) offset_set(p, mis, has_t);
      Particle pk0 = p;  // before the entrance kicks
      if (np) ab_kicks(p, kh, np);
      const Particle p_ph = p;  // the phase is taken here
      double phase = rf_phase(p, b[2], f, b[3]);
      // forward slices: K[i] = state before kick i, D[i] = state before drift i, phases
      Particle Kin[kAdjMaxSteps + 1], Din[kAdjMaxSteps];
      double ph[kAdjMaxSteps + 1];
      for (int i = 0; i <= n_slice; i++) {
        ph[i] = phase;
        Kin[i] = p;
        double dE = 1.0 * voltage * sin(phase) / n_slice;
        if (i == 0 || i == n_slice) dE = dE / 2;
        energy_kick(p, dE, G);
        if (i != n_slice) {
          refresh(p, G);
          Din[i] = p;
          double z = p.z;
          drift(p, slice_len);
          phase = phase + kTwoPi * f * (p.z - z) / (kCLight * p.beta);
        }
      }
      refresh(p, G);
      const Particle p_exit = p;  // before the exit kicks
      if (misal && has_t) vjp_tilt(mis[2], -mis[3], a);
      if (np) vjp_ab_kicks(p_exit, kh, np, a, gscale);
      double b_phase = 0;
      for (int i = n_slice; i >= 0; i--) {
        if (i != n_slice) {
          // phase_{i+1} = phase_i + 2 pi f (z_after - z_before) / (c beta), beta of Din[i]
          const Particle& d = Din[i];
          Particle e = d;
          drift(e, slice_len);
          double cfac = kTwoPi * f / (kCLight * d.beta);
          a.z += b_phase * cfac;                // through z_after (the drift's output)
          vjp_drift(d, slice_len, a, G);
          a.z += -b_phase * cfac;               // z_before
          a.beta += -b_phase * cfac * (e.z - d.z) / d.beta;
        }
        double dE = 1.0 * voltage * sin(ph[i]) / n_slice;
        double dEfac = 1.0 * voltage / n_slice;
        if (i == 0 || i == n_slice) {
          dE = dE / 2;
          dEfac = dEfac / 2;
        }
        double g_dE = 0;
        vjp_energy_kick(Kin[i], dE, a, g_dE, G);
        b_phase += g_dE * dEfac * cos(ph[i]);
      }
      // phase0 = modulo2(2 pi (phi0 - t f) + ..., pi), t = -z / (beta c)
      double dt_dz = -1 / (p_ph.beta * kCLight), dt_dbeta = p_ph.z / (p_ph.beta * p_ph.beta * kCLight);
      a.z += b_phase * (-kTwoPi * f) * dt_dz;
      a.beta += b_phase * (-kTwoPi * f) * dt_dbeta;
      if (np) vjp_ab_kicks(pk0, kh, np, a, gscale);
      if (misal && has_t) vjp_tilt(mis[2], mis[3], a);
      return;
    }
    default:
      return;  // marker
  }
}

// ---- per-particle driver: forward with checkpoints, then the reverse sweep -------------------
//
// Loss: sum over particles alive after n_turns of loss_scale * (x^2 + y^2). Buffers are
// structure-of-arrays with particle stride N: row r, component k of particle j at
// buf[(r * 7 + k) * N + j]. Checkpoints hold the state at the start of every `every`-th turn;
// in the reverse sweep each segment is re-run from its checkpoint storing the state at each turn
// start, and each turn is re-run storing every element's input, so the sweep runs backwards over
// elements with each element's input at hand (three levels: checkpoints, turns, elements).
struct AdjArgs {
  const EleHdr* hdr;
  const ApRec* ap;
  const double* pool;
  int32_t n_ele;
  int32_t n_turns;
  int32_t every;             // checkpoint interval in turns
  int64_t N;                 // particle stride of every buffer
  Globals G;
  const int32_t* param_of_ele;  // [n_ele]: gradient slot of the element, -1 if none
  double* ckpt;              // [ceil(n_turns / every)][7][N]
  double* turnbuf;           // [every][7][N]
  double* elebuf;            // [n_ele][7][N]
  double* gradbuf;           // [n_slots][N], accumulated (zeroed by the caller)
  double* lossbuf;           // [N]
  double* vec;               // [6][N] in/out
  double* beta;              // [N] in/out
  int32_t* state;            // [N] in/out
  double loss_scale;
};

BG_HD void adj_store(double* buf, int64_t row, int64_t N, int64_t j, const Particle& p) {
  double* q = buf + row * 7 * N + j;
  q[0] = p.x;
  q[N] = p.px;
  q[2 * N] = p.y;
  q[3 * N] = p.py;
  q[4 * N] = p.z;
  q[5 * N] = p.pz;
  q[6 * N] = p.beta;
}

BG_HD void adj_load(const double* buf, int64_t row, int64_t N, int64_t j, Particle& p, const Globals& G) {
  const double* q = buf + row * 7 * N + j;
  p.x = q[0];
  p.px = q[N];
  p.y = q[2 * N];
  p.py = q[3 * N];
  p.z = q[4 * N];
  p.pz = q[5 * N];
  p.beta = q[6 * N];
  p.state = S_ALIVE;
  refresh(p, G);
}

// One turn of track1 over every element; false if the particle was lost. The adjoint accepts no
// element with an extra block or a pitched offset (adj_supported), so the lean track1 serves.
BG_HD bool adj_turn(Particle& p, const AdjArgs& a, bool first_turn, double* store, int64_t j) {
  for (int ie = 0; ie < a.n_ele; ++ie) {
    if (store) adj_store(store, ie, a.N, j, p);
    if (track1<false>(p, a.hdr[ie], a.pool, a.ap, a.G, first_turn && ie == 0)) return false;
  }
  return true;
}

BG_HD void adj_particle(const AdjArgs& a, int64_t j) {
  const int64_t N = a.N;
  Particle p;
  p.x = a.vec[j];
  p.px = a.vec[N + j];
  p.y = a.vec[2 * N + j];
  p.py = a.vec[3 * N + j];
  p.z = a.vec[4 * N + j];
  p.pz = a.vec[5 * N + j];
  p.beta = a.beta[j];
  p.state = a.state[j];
  a.lossbuf[j] = 0;
  if (p.state != S_ALIVE) return;
  refresh(p, a.G);
  bool alive = true;
  for (int t = 0; t < a.n_turns && alive; ++t) {
    if (t % a.every == 0) adj_store(a.ckpt, t / a.every, N, j, p);
    alive = adj_turn(p, a, t == 0, nullptr, j);
  }
  a.vec[j] = p.x;
  a.vec[N + j] = p.px;
  a.vec[2 * N + j] = p.y;
  a.vec[3 * N + j] = p.py;
  a.vec[4 * N + j] = p.z;
  a.vec[5 * N + j] = p.pz;
  a.beta[j] = p.beta;
  a.state[j] = p.state;
  if (!alive) return;  // lost particles are outside the loss
  a.lossbuf[j] = a.loss_scale * (p.x * p.x + p.y * p.y);
  Adj lam = {2 * a.loss_scale * p.x, 0, 2 * a.loss_scale * p.y, 0, 0, 0, 0};
  const int n_seg = (a.n_turns + a.every - 1) / a.every;
  for (int seg = n_seg - 1; seg >= 0; --seg) {
    const int t0 = seg * a.every;
    const int nt = (a.n_turns - t0 < a.every) ? a.n_turns - t0 : a.every;
    Particle q;
    adj_load(a.ckpt, seg, N, j, q, a.G);
    for (int t = 0; t < nt; ++t) {
      adj_store(a.turnbuf, t, N, j, q);
      adj_turn(q, a, t0 + t == 0, nullptr, j);
    }
    for (int t = nt - 1; t >= 0; --t) {
      adj_load(a.turnbuf, t, N, j, q, a.G);
      adj_turn(q, a, t0 + t == 0, a.elebuf, j);
      for (int ie = a.n_ele - 1; ie >= 0; --ie) {
        Particle e;
        adj_load(a.elebuf, ie, N, j, e, a.G);
        double gs = 0;
        vjp_element(a.hdr[ie], a.pool, e, lam, gs, a.G);
        const int slot = a.param_of_ele[ie];
        if (slot >= 0) a.gradbuf[slot * N + j] += gs;
      }
    }
  }
}

}  // namespace bmadgpu
