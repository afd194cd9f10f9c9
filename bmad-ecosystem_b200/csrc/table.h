// table.h -- packed device element table, shared by the host packer (lattice.cpp) and the
// sm_100a kernels (track.cu).
//
// A lattice becomes one contiguous, 16-byte aligned byte image:
//   [EleHdr x n_ele][ApRec x n_ap][double pool]
// Each element header names its map kind, flags and the offset of its parameter block in the
// pool. Identical parameter blocks are stored once (a ring of identical FODO cells packs into a
// few hundred bytes). All per-element invariants (step lengths, bend-angle trig, edge-kick
// coefficients, scaled multipole coefficients, tilt cos/sin) are computed on the host, once.
#pragma once
#include <stdint.h>

namespace bmadgpu {

// Plain double for compile-time constants (stays double in the op-counting host build).
typedef double real_const;

enum Kind : uint8_t {
  K_MARKER = 0,  // no map (reference time only)
  K_DRIFT = 1,   // track_a_drift
  K_QUAD = 2,    // track_a_quadrupole
  K_THICK = 3,   // track_a_thick_multipole (sextupole, octupole, thick_multipole, monitor, ...)
  K_SBEND = 4,   // track_a_bend
  K_THIN = 5,    // multipole / ab_multipole thin kicks (track1_bmad.f90:142-166)
  K_RFCAV = 6    // track_a_rfcavity
};

enum Flag : uint16_t {
  F_MISALIGN = 1 << 0,     // straight offset + tilt transform around the body
  F_AP_ENTRANCE = 1 << 1,  // aperture checked at the entrance
  F_AP_EXIT = 1 << 2,      // aperture checked at the exit
  F_AP_ELLIPTICAL = 1 << 3,
  F_EDGE_IN = 1 << 4,      // sbend entrance edge kick (Hwang)
  F_EDGE_OUT = 1 << 5,     // sbend exit edge kick (Hwang)
  F_KICKS = 1 << 6,        // multipole kicks present
  F_BEND_K1 = 1 << 7,      // sbend body with k1 (sbend_body_with_k1_map)
  F_REF_ORB_N0 = 1 << 8,   // thin multipole: n = 0 as a zero-length bend (MAD convention)
  F_BEND_DRIFT = 1 << 9,   // sbend with g == 0 and dg == 0 or zero step: drift body
  F_ZERO_LEN = 1 << 10,    // element length is zero
  F_TILT = 1 << 11,        // misalign block carries a non-zero tilt rotation
  F_KICK_B_FROM2 = 1 << 12, // both kick arrays: every a_n zero and b_0 = b_1 = 0, at least 3 orders
  F_PITCH = 1 << 13,       // misalign block of the pitched form (straight elements) or the bend frame
  F_EXTRA = 1 << 14,       // extra block (EleHdr::extra): electric multipoles, higher-order edge fringes
  F_AP_WINDOW = 1 << 15    // the aperture record carries collimator phase-space windows
};

struct EleHdr {            // 16 bytes
  uint8_t kind;
  uint8_t n_pole;          // number of multipole orders kicked (ix_mag_max + 1), 0 = none
  uint16_t flags;
  uint16_t n_step;
  uint16_t ap_index;       // index into the aperture records
  uint32_t param;          // offset (in doubles) of the parameter block in the pool
  uint32_t extra;          // offset (in doubles) of the extra block (F_EXTRA), else 0
};

struct ApRec {             // 112 bytes
  // rectangular: the limits (x1_lim = -x1_limit, x2_lim = x2_limit, ...); elliptical: the
  // half widths and centres of elliptical_params_setup (x1_lim = x_width2, x2_lim = x0,
  // y1_lim = y_width2, y2_lim = y0)
  double x1_lim, x2_lim, y1_lim, y2_lim;
  // collimator phase-space windows (F_AP_WINDOW): half width and centre in px, py, z, pz
  double win[8];
  double win_kind;         // 1 ecollimator (elliptical px-py and z-pz windows), 2 rcollimator
  double pad;
};

// Parameter block layouts (indices in doubles from EleHdr::param).
// K_DRIFT:  [0] L
// K_QUAD:   [0] b1  [1] L  [2] step_len  then kicks, then misalign
// K_THICK:  [0] step_len  then kicks, then misalign
// K_SBEND:  [0] step_len [1] g [2] g_tot [3] dg [4] angle [5] cos_a [6] sin_a [7] sinc_a
//           [8] cosc_a [9] (g step_len)^2 sincc_a [10] k1 = b1/L [11] f_p0c = r_step p0c/(c q)
//           [12..18] entrance edge: gt gt2 gs2 k1_tane fg_factor g_tot gt*g_tot*(1+2tan^2)
//           [19..25] exit edge:     (same)
//           then kicks (bend form: plain b_n, a_n), then misalign (ref_tilt only: cos, sin)
// K_THIN:   per order n < n_pole: [knl, cos(tilt), sin(tilt), tilt == 0], then misalign
// K_RFCAV:  [0] voltage [1] rf_frequency [2] phi0 [3] twopi*phi0_multipass [4] slice_len
//           [5] n_slice  then kicks (half kicks 0.5*r_step), then misalign
// kicks: n_pole pairs for the end (half) kick followed, for K_QUAD/K_THICK, by n_pole pairs for
//        the interior (full) kick: (b_n*scale, a_n*scale), n = 0 .. n_pole-1.
// misalign: [x_off, y_off, cos_t, sin_t]; with F_PITCH (straight elements with x/y pitch or
//           z_offset) followed by [z_off, L/2, L/2 - 0, L/2 - L, 2 (L/2)] and the rotations W^-1
//           and W of floor_angles_to_w_mat(x_pitch, y_pitch, 0), row-major: 27 doubles
// bend frame (K_SBEND with F_MISALIGN | F_PITCH: offsets, pitches or z_offset on a bend), in
//           place of the misalign block: [n_set, n_unset, s_target set, s_target unset, W set (9),
//           W unset (9)] then n_set + n_unset steps of 16 doubles [op, v1 (3), M (9), v2 (3)]
//           acting on the position r = (x, y, 0): op & FS_SUB: r -= v1; FS_SUBZ: r_z -= v1_z;
//           FS_MAT: r = M r; FS_ADD: r += v2; FS_ADDZ: r_z += v2_z (in that order). W rotates the
//           momentum; the particle then drifts from r_z to s_target.
// extra block (F_EXTRA; quadrupole, sextupole, octupole, thick_multipole with electric multipoles
//           or an edge fringe, sbend with electric multipoles or fringe_type full):
//           [0] n_elec  [1] electric kick scale at the ends  [2] scale of the interior kicks
//           (step_len / 2 and step_len; bends step_len * 0.5 and step_len * 1.0)  [3] entrance
//           edge bits  [4] exit edge bits  [5] at_sign charge entrance  [6] at_sign charge exit
//           [7] mass / p0c  [8] hard-edge multipole order n (1 or 2)  [9] its strength (k1 or k2)
//           [10] k1 [11] fq1 [12] fq2 (soft quadrupole edge)  [13] g_tot [14] beta0 (exact bend
//           edge)  [15..17] entrance e1, fint, hgap  [18..20] exit e2, fintx, hgapx
//           elseparator: [21] steps through the separator field (kick != 0)  [22] cos, [23] sin
//           of the field angle atan2(vk, hk)  [24] angle != 0  [25] k_E = kick / l  [26] beta0
//           [27] (mass / p0c)^2  [28] at_sign charge p0c / l entrance  [29] the same, exit
//           [30] hkick [31] vkick
//           then (b_n, a_n) for n < n_elec (r0_elec scaled). Edge bits (EdgeBit): EX_CALL the
//           element's apply_element_edge_kick acts at this end (beta check), EX_ELEC the electric
//           longitudinal fringe, EX_HARD hard_multipole_edge_kick, EX_SOFT
//           soft_quadrupole_edge_kick, EX_EXACT exact_bend_edge_kick (in place of Hwang's), EX_ESEP
//           the elseparator's longitudinal fringe.
constexpr int SB_EDGE_IN = 12, SB_EDGE_OUT = 19, SB_FIXED = 26;
constexpr int EL_FIXED = 32, BF_FIXED = 22, BF_STEP = 16;
enum EdgeBit { EX_CALL = 1, EX_ELEC = 2, EX_HARD = 4, EX_SOFT = 8, EX_EXACT = 16, EX_ESEP = 32 };
enum FrameOp { FS_SUB = 1, FS_SUBZ = 2, FS_MAT = 4, FS_ADD = 8, FS_ADDZ = 16 };
constexpr int RF_FIXED = 6;

struct TableInfo {
  uint32_t n_ele;
  uint32_t n_ap;
  uint32_t hdr_bytes;      // n_ele * sizeof(EleHdr), 16-aligned
  uint32_t ap_bytes;       // n_ap * sizeof(ApRec)
  uint32_t pool_doubles;
  uint32_t total_bytes;    // whole image, 16-aligned
  double turn_ref_time;    // sum of delta_ref_time over the elements
  uint32_t rare;           // some element has an extra block or a pitched offset / bend frame
};

struct Globals {            // branch constants (lat_param_struct / bmad_com) and derived terms
  double p0c, e_tot, mass, beta0, max_ap;
  double mass2;             // mass**2
  double lez_b02;           // beta0**2           (low_energy_z_correction.f90:44)
  double lez_f;             // beta0**2 * (2 * beta0**2 - (mass / e_tot)**2 / 2)
  double lez_me2;           // (mass / e_tot)**2
  double lez_thresh;        // 3d-7 * e_tot
  double charge;            // charge_of(species)
  double inv_beta0;         // 1 / beta0 (rounded), the shared reciprocal of the quotients by beta0
};


// Signed binomial tables of c_multi.f90:38-63 (cm: no_n_fact = T, cf: c(n,m)), computed with the
// reference's operation sequence.
void build_cmulti_tables(double cm[22][22], double cf[22][22]);

}  // namespace bmadgpu
