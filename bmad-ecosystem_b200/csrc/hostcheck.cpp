// hostcheck.cpp -- TEST-ONLY host build of the device maps (elements.cuh, maps.cuh).
//
// Runs the exact per-particle element code of the sm_100a kernel on the CPU, so the tests can
// check the device algorithm against the oracle without a GPU and count its floating-point
// operations. It is built into a separate library (_build/libbmadgpu_hostcheck.so) that the
// product never loads; libbmadgpu.so has no CPU tracking path.

// The host build of the plain tracking kernel's maps, with its shared-reciprocal quotients.
#define BG_SHARED_RECIPROCAL
#include <cstring>
#include <string>

#include "../../include/bmadgpu.h"
#include "elements.cuh"
#include "lattice.h"

using namespace bmadgpu;

namespace bmadgpu {
double h_cmulti[kNPole][kNPole];
double h_cfull[kNPole][kNPole];
}

namespace {
thread_local std::string g_err;

Globals make_globals(const bmadgpu_param& p) {
  Globals g;
  g.p0c = p.p0c;
  g.e_tot = p.e_tot;
  g.mass = p.mass;
  g.beta0 = p.p0c / p.e_tot;
  g.max_ap = p.max_aperture_limit;
  g.mass2 = p.mass * p.mass;
  double me = p.mass / p.e_tot;
  g.lez_me2 = me * me;
  g.lez_b02 = g.beta0 * g.beta0;
  g.lez_f = g.lez_b02 * (2 * g.lez_b02 - g.lez_me2 / 2);
  g.lez_thresh = 3e-7 * p.e_tot;
  g.charge = p.charge;
  g.inv_beta0 = 1 / g.beta0;
  return g;
}
}  // namespace

extern "C" {

const char* bmadgpu_hostcheck_last_error(void) { return g_err.c_str(); }

// Tracks the bunch (host SoA) n_turns over all elements with the device element code.
int bmadgpu_hostcheck_track(const bmadgpu_element* eles, int32_t n_ele, const bmadgpu_param* param,
                            bmadgpu_bunch* b, int32_t n_turns) {
  static bool tables = false;
  if (!tables) {
    build_cmulti_tables(h_cmulti, h_cfull);
    tables = true;
  }
  PackedLattice pk;
  int r = pack_lattice(eles, n_ele, *param, pk, g_err);
  if (r) return r;
  const uint8_t* tbl = pk.image.data();
  const EleHdr* hdr = reinterpret_cast<const EleHdr*>(tbl);
  const ApRec* ap = reinterpret_cast<const ApRec*>(tbl + pk.info.hdr_bytes);
  const double* pool = reinterpret_cast<const double*>(tbl + pk.info.hdr_bytes + pk.info.ap_bytes);
  const Globals G = make_globals(*param);
  const int64_t n = b->n;
  for (int64_t j = 0; j < n; j++) {
    Particle p;
    p.x = b->vec[j]; p.px = b->vec[n + j]; p.y = b->vec[2 * n + j];
    p.py = b->vec[3 * n + j]; p.z = b->vec[4 * n + j]; p.pz = b->vec[5 * n + j];
    p.beta = b->beta[j];
    p.state = b->state[j];
    if (p.state != S_ALIVE) continue;
    refresh(p, G);
    int lost_loc = 0, lost_ele = -1, lost_turn = -1;
    for (int turn = 0; turn < n_turns && !lost_loc; turn++) {
      for (int ie = 0; ie < n_ele; ie++) {
        int loc = track1(p, hdr[ie], pool, ap, G, turn == 0 && ie == 0);
        if (loc) { lost_loc = loc; lost_ele = ie; lost_turn = turn; break; }
      }
    }
    b->vec[j] = p.x; b->vec[n + j] = p.px; b->vec[2 * n + j] = p.y;
    b->vec[3 * n + j] = p.py; b->vec[4 * n + j] = p.z; b->vec[5 * n + j] = p.pz;
    b->beta[j] = p.beta;
    b->state[j] = p.state;
    if (lost_loc) {
      if (b->ix_ele) b->ix_ele[j] = lost_ele;
      if (b->ix_turn) b->ix_turn[j] = lost_turn;
      if (b->location) b->location[j] = lost_loc;
    }
  }
  return 0;
}

}  // extern "C"
