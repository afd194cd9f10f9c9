// particle.cuh -- one particle's multi-turn loop, shared by the single-lattice kernel (k_track)
// and the batched kernel (k_batch_track) so that both do the same arithmetic.
//
// The loop is the element loop of track_bunch (bmad/multiparticle/beam_mod.f90:159-166) inside
// the turn loop of ltt_run_beam_mode (bsim/modules/lt_tracking_mod.f90:1631-1713), with track1
// (elements.cuh) around each element. A lost particle leaves at once and records where it was
// lost as track1_bunch_hom leaves it (bmad/multiparticle/beam_utils.f90:81-86).
#pragma once
#include "elements.cuh"

namespace bmadgpu {

// Structure-of-arrays particle storage: coordinate i of particle j is vec[i * ld + j].
struct SoA {
  double* vec;
  double* beta;
  double* t;          // nullable
  int32_t* state;
  int32_t* ix_ele;    // nullable
  int32_t* ix_turn;   // nullable
  int32_t* location;  // nullable
  int64_t ld;
};

__device__ __forceinline__ void load_hdr(const EleHdr* hdr, int i, EleHdr& h) {
  uint4 raw = *reinterpret_cast<const uint4*>(hdr + i);
  h = *reinterpret_cast<const EleHdr*>(&raw);
}

struct LossInfo {
  int loc = 0, ele = -1, turn = -1;  // coord%location, element and turn of the loss
};

__device__ __forceinline__ void load_particle(const SoA& s, int64_t j, Particle& p) {
  const int64_t ld = s.ld;
  p.x = s.vec[j];
  p.px = s.vec[ld + j];
  p.y = s.vec[2 * ld + j];
  p.py = s.vec[3 * ld + j];
  p.z = s.vec[4 * ld + j];
  p.pz = s.vec[5 * ld + j];
  p.beta = s.beta[j];
  p.state = s.state[j];
}

// One turn over elements [ix_start, ix_end). Returns false (and fills li) if the particle is lost.
template <bool FULL = true>
__device__ __forceinline__ bool track_turn(Particle& p, const EleHdr* __restrict__ hdr, const double* __restrict__ pool,
                                           const ApRec* __restrict__ ap, const Globals& G, int ix_start, int ix_end,
                                           bool first_turn, int turn_no, LossInfo& li) {
  for (int ie = ix_start; ie < ix_end; ++ie) {
    EleHdr h;
    load_hdr(hdr, ie, h);
    int loc = track1<FULL>(p, h, pool, ap, G, first_turn && ie == ix_start);
    if (loc) {
      li.loc = loc;
      li.ele = ie;
      li.turn = turn_no;
      return false;
    }
  }
  return true;
}

// Writes a particle back after a launch of n_turns turns starting at turn turn0. Particles that
// were not alive at the start (li.loc == 0 and !alive) are left untouched. The time coordinate
// follows from the reference time elapsed: t + z/(beta c) advances by delta_ref_time in every
// element (track_a_*: orbit%t update); ref_prefix[i] = sum of delta_ref_time over elements < i and
// seg_ref = ref_prefix[ix_end] - ref_prefix[ix_start] is one turn's share.
__device__ __forceinline__ void store_particle(const SoA& s, int64_t j, const Particle& p, bool alive,
                                               const LossInfo& li, double z_in, double beta_in, int n_turns,
                                               int turn0, double seg_ref, const double* __restrict__ ref_prefix,
                                               int ix_start) {
  if (!(alive || li.loc)) return;
  const int64_t ld = s.ld;
  s.vec[j] = p.x;
  s.vec[ld + j] = p.px;
  s.vec[2 * ld + j] = p.y;
  s.vec[3 * ld + j] = p.py;
  s.vec[4 * ld + j] = p.z;
  s.vec[5 * ld + j] = p.pz;
  s.beta[j] = p.beta;
  s.state[j] = p.state;
  if (s.t && beta_in > 0) {
    double elapsed = alive ? n_turns * seg_ref : (li.turn - turn0) * seg_ref + (ref_prefix[li.ele] - ref_prefix[ix_start]);
    double tb = (p.beta > 0) ? p.z / (p.beta * kCLight) : 0.0;
    s.t[j] = s.t[j] + (z_in / (beta_in * kCLight) + elapsed - tb);
  }
  if (!alive) {
    if (s.ix_ele) s.ix_ele[j] = li.ele;
    if (s.ix_turn) s.ix_turn[j] = li.turn;
    if (s.location) s.location[j] = li.loc;
  }
}

}  // namespace bmadgpu
