// elements.cuh -- per-element bodies and the track1 wrapper (shared by the kernels and the
// test-only host check build).
#pragma once
#include "maps.cuh"

namespace bmadgpu {

// ---- element bodies (track1_bmad dispatch, bmad/low_level/track1_bmad.f90:64-272) ----------

// Each body and track1 come in two forms: FULL = true handles every element form; FULL = false,
// for tables without any extra block or pitched offset (TableInfo::rare = 0, the common rings),
// leaves those forms out, so that their out-of-line helpers add nothing to the kernels that
// track such rings.
template <bool FULL>
BG_HD void body_quad(Particle& p, const EleHdr& h, const double* __restrict__ b, const double* __restrict__ el,
                     const Globals& G) {
  // track_a_quadrupole, bmad/low_level/track_a_quadrupole.f90; the kick before the body and the
  // kick after each step share one call site. With an extra block (F_EXTRA) the edges carry the
  // hard/soft quadrupole fringe and the electric fringe, and with electric multipoles every
  // magnetic kick is followed by the electric one.
  const int np = h.n_pole;
  const double* kh = b + 3;
  const double* kf = kh + 2 * np;
  const double* mis = b + 3 + 4 * np;
  const bool has_t = h.flags & F_TILT;
  const double* xb = (FULL && (h.flags & F_EXTRA)) ? el : nullptr;
  const bool elec = xb && xb[0] != 0;
  const bool pitched = FULL && (h.flags & F_PITCH);
  if (h.flags & F_MISALIGN) offset_set(p, mis, has_t, pitched);
  if (xb) {
    straight_edge(p, xb, true, G);
    if (p.state != S_ALIVE) return;
  }
  const double b1 = b[0], length = b[1], step_len = b[2];
  const int n_step = h.n_step;
  const bool b_from2 = h.flags & F_KICK_B_FROM2;
  for (int i = 0; i <= n_step; i++) {
    if (i > 0) quad_step(p, b1, length, step_len, G);
    const bool end = (i == 0 || i == n_step);
    if (np) ab_kicks(p, end ? kh : kf, np, b_from2);
    if (elec) elec_kicks(p, el, end ? el[1] : el[2], G);
  }
  if (xb) {
    straight_edge(p, xb, false, G);
    if (p.state != S_ALIVE) return;
  }
  if (h.flags & F_MISALIGN) offset_unset(p, mis, has_t, pitched);
}

template <bool FULL>
BG_HD void body_thick(Particle& p, const EleHdr& h, const double* __restrict__ b, const double* __restrict__ el,
                      const Globals& G) {
  // track_a_thick_multipole, bmad/low_level/track_a_thick_multipole.f90:18-133
  const int np = h.n_pole;
  const double* kh = b + 1;
  const double* kf = kh + 2 * np;
  const double* mis = b + 1 + 4 * np;
  const bool has_t = h.flags & F_TILT;
  const double* xb = (FULL && (h.flags & F_EXTRA)) ? el : nullptr;
  const bool elec = xb && xb[0] != 0;
  const bool elsep = xb && xb[21] != 0;   // elseparator field steps
  const bool pitched = FULL && (h.flags & F_PITCH);
  Particle start;
  if (elsep) start = p;
  if (h.flags & F_MISALIGN) offset_set(p, mis, has_t, pitched);
  if (xb) {
    straight_edge(p, xb, true, G);
    if (p.state != S_ALIVE) return;
  }
  const double step_len = b[0];
  const int n_step = h.n_step;
  const bool b_from2 = h.flags & F_KICK_B_FROM2;
  for (int i = 0; i <= n_step; i++) {
    if (i > 0) {
      if (elsep) {
        if (!elsep_step(p, xb, step_len, start, G)) return;
      } else {
        drift(p, step_len);
      }
    }
    const bool end = (i == 0 || i == n_step);
    if (np) ab_kicks(p, end ? kh : kf, np, b_from2);
    if (elec) elec_kicks(p, el, end ? el[1] : el[2], G);
  }
  if (xb) {
    straight_edge(p, xb, false, G);
    if (p.state != S_ALIVE) return;
  }
  if (h.flags & F_MISALIGN) offset_unset(p, mis, has_t, pitched);
}

BG_HD void bend_kick(Particle& p, const double* __restrict__ b, int np, const double* __restrict__ el, bool half,
                     const Globals& G) {
  // apply_multipole_kicks (exact_multipoles = off), track_a_bend.f90:338-471: both fields from
  // the incoming orbit, then the magnetic kick, then the electric one (el, when present)
  double B1 = 0, B2 = 0, E1 = 0, E2 = 0;
  const double coef = half ? 0.5 : 1.0;
  if (np) ab_field(p, b + SB_FIXED, np, b[11], B1, B2);
  if (el) elec_field(p, el, E1, E2);
  if (np) {
    double f_coef = coef * G.charge * (1 + b[1] * p.x) * kCLight / G.p0c;
    p.px = p.px - f_coef * B2;
    p.py = p.py + f_coef * B1;
  }
  if (el) bend_elec_kick(p, el, half ? el[1] : el[2], b[1], E1, E2, G);
}

template <bool FULL>
BG_HD void body_bend(Particle& p, const EleHdr& h, const double* __restrict__ b, const double* __restrict__ el,
                     const Globals& G) {
  // track_a_bend, bmad/low_level/track_a_bend.f90:18-333
  const int np = h.n_pole;
  const double* mis = b + SB_FIXED + 2 * np;
  const double* xb = (FULL && (h.flags & F_EXTRA)) ? el : nullptr;   // electric multipoles / fringe_type full
  const double* e = (xb && xb[0] != 0) ? xb : nullptr;      // electric multipoles
  const int in = xb ? (int)xb[3] : 0, out = xb ? (int)xb[4] : 0;
  if (h.flags & F_MISALIGN) {
    if (FULL && (h.flags & F_PITCH)) bend_frame(p, mis, true);   // offsets / pitches: the bend frame
    else tilt(p, mis[2], mis[3]);                     // ref_tilt only, offset_particle.f90:263-266
  }
  // apply_element_edge_kick at the entrance (bend_edge_kick, fringe_mod.f90:40-128): hard-edge
  // multipole, then the exact (fringe_type full) or Hwang edge, then the electric fringe
  if ((in & EX_CALL) && p.beta == 0) p.state = S_LOST;
  if (in & EX_HARD) hard_edge(p, xb, true);
  if (in & EX_EXACT) exact_bend_edge(p, xb, true);
  else if (h.flags & F_EDGE_IN) hwang_edge(p, b + SB_EDGE_IN, true);
  if (in & EX_ELEC) elec_fringe(p, xb, xb[5], G);
  if (orbit_too_large(p, G)) return;
  if (np || e) bend_kick(p, b, np, e, true, G);
  for (int n = 1; n <= h.n_step; n++) {
    if (h.flags & F_BEND_K1) {
      bend_k1_step(p, b);
      p.z = p.z + low_energy_z(p, b[0], G);
    } else if (h.flags & F_BEND_DRIFT) {
      drift(p, b[0]);
    } else {
      if (!bend_exact_step(p, b, G)) return;
    }
    if (np || e) bend_kick(p, b, np, e, n == h.n_step, G);
  }
  if (orbit_too_large(p, G)) return;
  // at the exit: the electric fringe, then the exact or Hwang edge, then the hard-edge multipole
  if ((out & EX_CALL) && p.beta == 0) p.state = S_LOST;
  if (out & EX_ELEC) elec_fringe(p, xb, xb[6], G);
  if (out & EX_EXACT) exact_bend_edge(p, xb, false);
  else if (h.flags & F_EDGE_OUT) hwang_edge(p, b + SB_EDGE_OUT, false);
  if (out & EX_HARD) hard_edge(p, xb, false);
  if (h.flags & F_MISALIGN) {
    if (FULL && (h.flags & F_PITCH)) bend_frame(p, mis, false);
    else tilt(p, mis[2], -mis[3]);
  }
}

BG_HD void body_thin(Particle& p, const EleHdr& h, const double* __restrict__ b) {
  // multipole / ab_multipole, track1_bmad.f90:142-166 with multipole_kicks (multipole_mod.f90:32-51).
  // Block: per order n < n_pole: [knl, cos(tilt), sin(tilt), tilt == 0]; then misalign.
  const int np = h.n_pole;
  const double* mis = b + 4 * np;
  if (h.flags & F_MISALIGN) offset_set(p, mis, false);
  for (int n = 0; n < np; n++) {
    const double* q = b + 4 * n;
    double knl = q[0];
    if (knl == 0) continue;
    if (n == 0 && (h.flags & F_REF_ORB_N0)) {  // multipole_mod.f90:250-255
      double c = q[1], s = q[2];
      double x = p.x, y = p.y;
      p.px = p.px + 1.0 * knl * c * p.pz;
      p.py = p.py + 1.0 * knl * s * p.pz;
      p.z = p.z - 1.0 * knl * (c * x + s * y);
      continue;
    }
    thin_kick(p, knl, n, q[3] != 0, q[1], q[2]);
  }
  if (h.flags & F_MISALIGN) offset_unset(p, mis, false);
}

template <bool FULL>
BG_HD void body_rf(Particle& p, const EleHdr& h, const double* __restrict__ b, const Globals& G) {
  // track_a_rfcavity, bmad/low_level/track_a_rfcavity.f90:17-146 (relative time tracking)
  const int np = h.n_pole;
  const double* kh = b + RF_FIXED;
  const double* mis = kh + 2 * np;
  const bool has_t = h.flags & F_TILT;
  const bool pitched = FULL && (h.flags & F_PITCH);
  if (h.flags & F_MISALIGN) offset_set(p, mis, has_t, pitched);
  if (np) ab_kicks(p, kh, np);
  const double voltage = b[0], f = b[1], slice_len = b[4];
  const int n_slice = h.n_step;
  double phase = rf_phase(p, b[2], f, b[3]);
  for (int i = 0; i <= n_slice; i++) {
    double dE = 1.0 * voltage * m_sin(phase) / n_slice;
    if (i == 0 || i == n_slice) dE = dE / 2;
    energy_kick(p, dE, G);
    if (p.pz == -1) {
      p.state = S_LOST_PZ;
      return;
    }
    if (i != n_slice) {
      refresh(p, G);
      double z = p.z;
      drift(p, slice_len);
      phase = phase + kTwoPi * f * (p.z - z) / (kCLight * p.beta);
    }
  }
  refresh(p, G);
  if (np) ab_kicks(p, kh, np);
  if (h.flags & F_MISALIGN) offset_unset(p, mis, has_t, pitched);
}

// track1 around one element: entrance orbit/aperture checks, body, exit checks
// (track1.f90:179-196, 221-236, 289-329). Returns 0 if the particle survived, else its
// coord%location at the loss. The entrance orbit_too_large test repeats the previous element's
// exit test on unchanged coordinates, so it runs only for the first element of a launch.
template <bool FULL = true>
BG_HD int track1(Particle& p, const EleHdr& h, const double* __restrict__ pool,
                                      const ApRec* __restrict__ ap, const Globals& G, bool entry_check) {
  if (entry_check && orbit_too_large(p, G)) return L_UPSTREAM;
  const bool windows = FULL && (h.flags & F_AP_WINDOW);
  if (h.flags & F_AP_ENTRANCE) {
    aperture(p, ap[h.ap_index], h.flags & F_AP_ELLIPTICAL, windows);
    if (p.state != S_ALIVE) return L_UPSTREAM;
  }
  const double* b = pool + h.param;
  const double* el = pool + h.extra;
  switch (h.kind) {
    case K_DRIFT: drift(p, b[0]); break;
    case K_QUAD: body_quad<FULL>(p, h, b, el, G); break;
    case K_THICK: body_thick<FULL>(p, h, b, el, G); break;
    case K_SBEND: body_bend<FULL>(p, h, b, el, G); break;
    case K_THIN: body_thin(p, h, b); break;
    case K_RFCAV: body_rf<FULL>(p, h, b, G); break;
    default: break;  // K_MARKER
  }
  if (orbit_too_large(p, G)) return L_UPSTREAM;
  if (p.state != S_ALIVE) return L_INSIDE;
  if (h.flags & F_AP_EXIT) {
    aperture(p, ap[h.ap_index], h.flags & F_AP_ELLIPTICAL, windows);
    if (p.state != S_ALIVE) return L_DOWNSTREAM;
  }
  return 0;
}

}  // namespace bmadgpu
