/*
 * bmad_oracle.h -- CPU ORACLE (test infrastructure only; never the product path).
 *
 * A scalar C++ restatement of Bmad's bmad_standard single-particle tracking
 * (bmad/code/track1.f90 -> bmad/low_level/track1_bmad.f90 -> track_a_*) and of the OpenMP
 * bunch loop (bmad/multiparticle/beam_utils.f90:81-86). Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load it, and only to check the device results.
 *
 * Parity pinning: the element maps are checked against the Bmad_Standard golden lines of
 * regression_tests/tracking_method_test/output.correct and against
 * regression_tests/fringe_test/output.correct (tests/golden/). Multi-turn ring tracking has no
 * golden vectors in the reference (parity for multi-turn tracking is pinned element-wise only).
 *
 * Arithmetic: double (Fortran real(rp)); the particle time coord%t and the RF time use
 * __float128 as the reference's real(qp) does (bmad_struct.f90:554, particle_rf_time.f90:45).
 * Built with -O2 -ffp-contract=off so no FMA contraction alters the Fortran operation order.
 */
#ifndef BMAD_ORACLE_H
#define BMAD_ORACLE_H

#include <stdint.h>
#include "bmadgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One particle, the coord_struct fields the path reads or writes (bmad_struct.f90:551-579). */
typedef struct oracle_coord {
  double vec[6];
  double beta;
  double p0c;
  double s;
  double t;          /* FP64 copy of the internal real(qp) time (see oracle_coord_t_qp) */
  double phase1;     /* coord%phase(1), written by rfcavity tracking */
  int32_t state;
  int32_t location;
  int32_t ix_ele;
  int32_t direction; /* must be +1 */
  int32_t time_dir;  /* must be +1 */
  int32_t pad;
  /* internal quad-precision time: 16 bytes, little-endian __float128 */
  unsigned char t_qp[16];
} oracle_coord;

/* Resolve bookkeeping (tilt_tot, has_misalign, ds_step/num_steps) of one element the way
 * attribute_bookkeeper.f90:146-170, 292-400 does; returns resolved num_steps or <0 on error. */
int32_t oracle_element_num_steps(const bmadgpu_element* ele, const bmadgpu_param* param);

/* init_coord for a bmad_standard particle at the upstream end of an element (beta from pz,
 * t = -z/(beta c)), init_coord.f90 lines covering orb%beta and orb%t. */
void oracle_init_coord(oracle_coord* orb, const double vec[6], const bmadgpu_param* param);

/* track1 (track1.f90:44-343) through one element. Returns 0, or a negative BMADGPU_E* code
 * for element types/flags this restatement does not cover. */
int oracle_track1(oracle_coord* orb, const bmadgpu_element* ele, int32_t ix_ele,
                  const bmadgpu_param* param);

/* hwang_bend_edge_kick (fringe_mod.f90:241-419) with make_matrix = T.
 * particle_at: 11 = first_track_edge$, 12 = second_track_edge$. mat6 is 6x6 row-major
 * (mat6[i*6+j] = Fortran mat6(i+1, j+1)), premultiplied by the edge matrix. */
/* offset_particle (bmad/code/offset_particle.f90:66-530) of one element, set (1) or unset (0),
 * drifting to the element's end, set_tilt and set_hvkicks true. */
int oracle_offset_particle(const bmadgpu_element* ele, const bmadgpu_param* param, int32_t set, oracle_coord* c);

/* check_aperture_limit (bmad/low_level/check_aperture_limit.f90:30-387) of one element at
 * particle_at (11 first_track_edge, 12 second_track_edge) on the coordinate c: its state after the
 * check and param%unstable_factor. */
int oracle_check_aperture(const bmadgpu_element* ele, const bmadgpu_param* param, int32_t particle_at,
                          oracle_coord* c, double* unstable_factor);

int oracle_hwang_bend_edge_kick(const bmadgpu_element* ele, const bmadgpu_param* param,
                                int32_t particle_at, oracle_coord* orb, double* mat6);

/* Ring tracking over n_turns x elements [0, n_ele), particle-parallel with OpenMP
 * (n_threads <= 0: all cores), element-outer as track_bunch/track1_bunch_hom are
 * (beam_mod.f90:159-166, beam_utils.f90:81-86). SoA arrays as in bmadgpu_bunch.
 * moments: NULL or [n_turns * 28] (n_live, sums of vec_i, sums of vec_i*vec_j, i<=j). */
int oracle_track_ring(const bmadgpu_element* eles, int32_t n_ele, const bmadgpu_param* param,
                      bmadgpu_bunch* bunch, int32_t turn0, int32_t n_turns, int32_t n_threads,
                      double* moments);

/* Number of OpenMP threads the oracle would use with n_threads <= 0. */
int32_t oracle_max_threads(void);

/* The eight libm functions the restated routines call (sin, cos, asin, atan2, sinh, cosh, exp,
 * tan; atan(v) is atan2(v, 1)): by default the host's; the given ones if all eight are non-NULL;
 * the host's again if any is NULL. Not thread-safe against a tracking call in progress. */
void oracle_set_libm(double (*f_sin)(double), double (*f_cos)(double), double (*f_asin)(double),
                     double (*f_atan2)(double, double), double (*f_sinh)(double), double (*f_cosh)(double),
                     double (*f_exp)(double), double (*f_tan)(double));

#ifdef __cplusplus
}
#endif

#endif
